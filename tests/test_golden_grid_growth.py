"""Grid-based growth (growth type 3) pinned against the reference's own output.

tests/golden/run07007_grid_growth.npz comes from the reference's no-Pardiso regression run 07007
(made by tests/golden/make_run07007_grid_growth.py): a three-layer rectangle with explicit ECM and
actin grown by two grid functions (nearest-corner interpolation, grids pinned on the initial mesh,
z range 0.5-1: a z function from 120 s and an x, y function from 60 s, both until 300 s) for 11
steps of 60 s. The run's log holds the diagonal of every grid-growth increment it made, step by
step, function by function in input order, element by element, to six significant digits.

The model-input reader (grid files read as the reference reads them, pinned relative positions,
relative heights, ECM and actin flags) with the oracle's restatement must produce the same
increments for the same elements in the same order (the reference logs the increment of every
element the function applies to), to the log's six digits. The device kernel must then produce the
oracle's increments - and the growth tensors they compose into - to 1e-12, for this run and for
bilinear interpolation with orientation angles on random grids.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import mesh
from tissueorigami_b200 import modelinput as MI

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run07007_grid_growth.npz")


def _setup():
    z = np.load(GOLDEN)
    entries = MI.parse(" ".join(str(t) for t in z["modelinput_tokens"]))
    files = {str(n): str(t) for n, t in zip(z["grid_names"], z["grid_texts"])}
    conn = z["conn"].astype(np.int32)
    place, spans = MI._element_placement(conn, z["place"])
    ecm = (place == MI.BASAL) | ((place == MI.MID) & spans)
    actin = (place == MI.APICAL) | (place == MI.APICAL_BULK) | ((place == MI.MID) & spans)
    funcs = []
    for gtype, g in MI.growth_blocks(entries):
        assert gtype == 3
        gm = MI._Entries(g)
        rates, angles = MI.read_growth_grid(files[gm.get("Filename(full-path)")[0]])
        zr = gm.num("zRange", n=2)
        funcs.append({"t0": float(np.float32(gm.num("InitialTime(sec)"))), "t1": float(np.float32(gm.num("FinalTime(sec)"))),
                      "rates": rates, "angles_deg": angles, "zmin": zr[0], "zmax": zr[1], "nx": rates.shape[0],
                      "ny": rates.shape[1], "flags": int(gm.flag("ApplyToColumnarLayer(bool)"))})
    state = MI.grid_element_state(z["x"], conn, z["place"], z["ttype"], place, spans, ecm, actin)
    interp = int(MI._Entries(entries).num("GridGrowthsInterpolationType(0=step,1=linear)"))
    dt = float(MI._Entries(entries).num("TimeStep(sec)"))
    return z, funcs, state, interp, dt


def test_fixture_is_what_the_reference_logged():
    z, funcs, state, interp, dt = _setup()
    assert [f["t0"] for f in funcs] == [120.0, 60.0] and [f["t1"] for f in funcs] == [300.0, 300.0]
    assert interp == 0 and dt == 60.0
    # the x, y function alone at 60 s, both functions at 120-240 s, none afterwards
    assert list(z["counts"]) == [0, 16, 32, 32, 32, 0, 0, 0, 0, 0, 0]


def test_oracle_grid_increments_match_the_reference_log():
    z, funcs, state, interp, dt = _setup()
    rel_pos, rel_z, eflags = state
    start = 0
    for t, n in zip(z["times"], z["counts"]):
        _, applied, inc = O.grid_growth_increments(funcs, rel_pos, rel_z, eflags, interp, float(t), dt, per_function=True)
        seq = [inc[f, e].reshape(3, 3).diagonal() for f in range(len(funcs)) for e in range(rel_z.shape[0])
               if applied[f, e]]
        logged = z["increments"][start:start + n]
        start += n
        assert len(seq) == n, (t, len(seq), n)
        if n:
            np.testing.assert_allclose(np.array(seq), logged, rtol=1e-6, atol=0)
    assert start == z["increments"].shape[0]


def test_oracle_grid_growth_composes_into_fg():
    """tfo_grow applies the grid increments after the uniform one: with no uniform growth and a
    tissue that does not move, Fg after each step is the product of the steps' increments."""
    z, funcs, state, interp, dt = _setup()
    rel_pos, rel_z, eflags = state
    conn = z["conn"].astype(np.int32)
    E = conn.shape[0]
    t = mesh.Tissue("run07007", conn, z["xref"], z["x"], np.ones(E), np.ones(E), np.zeros(E),
                    np.ones((z["x"].shape[0], 3), np.uint8), np.zeros((z["x"].shape[0], 3)), np.zeros(E, np.uint8),
                    np.zeros(E, np.uint8), np.zeros((E, 3)), np.zeros(E), z["place"].astype(np.int32),
                    z["circ"].astype(np.int32), dt=dt)
    fg = t.fg.copy()
    want = np.tile(np.eye(3), (E, 1, 1))
    for time in z["times"]:
        inc = O.grid_growth_increments(funcs, rel_pos, rel_z, eflags, interp, float(time), dt)
        fg, _, _, rot = O.grow(t, t.x, fg, grid_inc=inc)
        assert not rot.any()
        want = inc.reshape(-1, 3, 3) @ want
        np.testing.assert_allclose(fg.reshape(-1, 3, 3), want, rtol=0, atol=1e-15)


def _random_grids(rng, n_funcs=3):
    funcs = []
    for f in range(n_funcs):
        nx, ny = int(rng.integers(3, 9)), int(rng.integers(3, 7))
        rates = rng.uniform(-2e-4, 4e-4, (nx, ny, 3))
        angles = rng.uniform(-180.0, 360.0, (nx, ny))
        rates[0, 0, 1] = rates[0, 0, 0]  # an aspect ratio of 1: that corner's angle is left out
        funcs.append({"t0": 0.0, "t1": 1e9, "rates": rates, "angles_deg": angles, "zmin": 0.0, "zmax": 1.0,
                      "nx": nx, "ny": ny, "flags": 1})
    return funcs


def _bilinear_literal(f, rx, ry, dt):
    """Nearest-free restatement of one bilinear grid increment for one element (GrowthFunctionTypes.h
    :368-531 compatible angles, ShapeBase.cpp:545-655 interpolation), loop by loop in Python."""
    nx, ny = f["nx"], f["ny"]
    px, py = rx * float(np.float32(nx - 1)), ry * float(np.float32(ny - 1))
    ix, iy = int(np.floor(px)), int(np.floor(py))
    fx, fy = px - ix, py - iy
    if ix >= nx - 1:
        ix, fx = nx - 2, 1.0
    elif ix < 0:
        ix, fx = 0, 0.0
    if iy >= ny - 1:
        iy, fy = ny - 2, 1.0
    elif iy < 0:
        iy, fy = 0, 0.0
    corners = [(ix, iy), (ix + 1, iy), (ix, iy + 1), (ix + 1, iy + 1)]
    g = [list(f["rates"][i, j]) for i, j in corners]
    a, el = [0.0] * 4, [False] * 4
    for q, (i, j) in enumerate(corners):
        ar = abs(f["rates"][i, j, 0] / f["rates"][i, j, 1])
        ar = 1 / ar if ar < 1.0 else ar
        if ar < 1.1:
            el[q] = True
        else:
            a[q] = f["angles_deg"][i, j] * np.pi / 180.0
    for q in range(4):
        while a[q] < 0:
            a[q] += np.pi
        while a[q] > np.pi:
            a[q] -= np.pi
    kept = [q for q in range(4) if not el[q]]
    sel, tet = (kept[0], a[kept[0]]) if kept else (3, 0.0)
    for q in range(sel, 4):
        d = a[q] - tet
        turns = [(np.pi / 4, 3 * np.pi / 4, -np.pi / 2, True), (3 * np.pi / 4, 5 * np.pi / 4, -np.pi, False),
                 (5 * np.pi / 4, 7 * np.pi / 4, -1.5 * np.pi, True), (7 * np.pi / 4, np.inf, -2 * np.pi, False)]
        for lo, hi, shift, flip in turns:
            if (d > 0 and lo <= d < hi) or (d < 0 and -hi < d <= -lo):
                a[q] += shift if d > 0 else -shift
                if flip:
                    g[q][0], g[q][1] = g[q][1], g[q][0]
                break
    w = [(1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy]
    gone = sum(wq for wq, e in zip(w, el) if e)
    ang = sum(aq * wq for aq, wq in zip(a, w))
    if gone > 0:
        ang = 0.0 if gone >= 0.9999999 else ang / (1 - gone)
    grow = [sum(g[q][k] * w[q] for q in range(4)) for k in range(3)]
    D = np.diag(np.exp(np.array(grow) * dt))
    c, s = np.cos(ang), np.sin(ang)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    return D if ang == 0.0 else R @ D @ R.T


def test_oracle_bilinear_grid_matches_a_literal_restatement():
    rng = np.random.default_rng(3)
    funcs = _random_grids(rng, 1)
    E = 200
    rel_pos = rng.uniform(-0.05, 1.05, (E, 2))
    rel_z = np.full(E, 0.5)
    eflags = np.zeros(E, np.int32)
    inc = O.grid_growth_increments(funcs, rel_pos, rel_z, eflags, 1, 0.0, 60.0).reshape(-1, 3, 3)
    for e in range(E):
        np.testing.assert_allclose(inc[e], _bilinear_literal(funcs[0], rel_pos[e, 0], rel_pos[e, 1], 60.0),
                                   rtol=0, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["run07007", "bilinear"])
def test_device_grid_growth_matches_oracle(case):
    from tissueorigami_b200 import capi
    from tissueorigami_b200.newton import NewtonRaphsonSolver

    if case == "run07007":
        z, funcs, state, interp, dt = _setup()
        times = [float(v) for v in z["times"]]
        t = mesh.Tissue("run07007", z["conn"].astype(np.int32), z["xref"], z["x"], *mesh.lame(np.full(48, 100.0), 0.29),
                        np.zeros(48), np.ones((60, 3), np.uint8), np.zeros((60, 3)), np.zeros(48, np.uint8),
                        np.zeros(48, np.uint8), np.zeros((48, 3)), np.zeros(48), z["place"].astype(np.int32),
                        z["circ"].astype(np.int32), dt=dt)
    else:
        rng = np.random.default_rng(4)
        t = mesh.small_rectangle(nx=12, ny=7)
        t.fixed[:] = 1
        t.rates[:] = 0.0
        funcs = _random_grids(rng, 3)
        funcs[1]["t0"], funcs[2]["t1"] = 120.0, 180.0
        funcs[0]["zmin"] = 0.6  # outside this single-layer tissue's relative height 0.5
        funcs[0]["zmax"] = 1.0
        place, spans = MI._element_placement(t.conn, t.node_placement)
        state = MI.grid_element_state(t.x, t.conn, t.node_placement, np.zeros(t.n_nodes, np.int32), place, spans,
                                      np.zeros(t.n_elems, bool), np.zeros(t.n_elems, bool))
        interp, dt = 1, t.dt
        times = [k * dt for k in range(5)]
    with NewtonRaphsonSolver.from_tissue(t) as s:
        s.set_grid_growth(funcs, interp, *state)
        s.set_time(times[0])
        fg = t.fg.copy()
        x = t.x.copy()
        for time in times:
            assert s.time() == time
            inc = O.grid_growth_increments(funcs, *state, interp, time, dt)
            fg, _, _, _ = O.grow(t, t.x, fg, grid_inc=inc)
            x, rc, _ = s.runOneStep(x, dt)
            assert rc == capi.TF_OK
            fg_dev, _ = s.get_growth()
            err = np.abs(fg_dev.reshape(-1, 9) - fg).max() / np.abs(fg).max()
            assert err <= 1e-12, (case, time, err)
        np.testing.assert_array_equal(x, t.x)  # every DoF fixed: no node moved
