"""The model-input loader (tissueorigami_b200.modelinput) on the reference's own input.

The Pardiso regression run 07008 of the reference recorded the set-up it derived from its
model input - Young's modulus per element, external viscosity per node, the binding pairs, the
ECM elements - and its first step's positions (tests/golden/run07008_newton_step1.npz, with the
model input file's tokens). The loader must derive the same set-up from the same model input
and mesh by the reference's rules, and that set-up must give the recorded first step.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import modelinput as MI

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run07008_newton_step1.npz")


def _load():
    z = np.load(GOLDEN)
    text = " ".join(str(t) for t in z["modelinput_tokens"])
    st = MI.setup(MI.parse(text), (z["x"], z["place"], z["ttype"], z["circ"], z["conn"], z["xref"]))
    return st, z


def test_parse_keeps_keys_values_and_order():
    e = MI.parse("Sec:\n  A(x): 1 2 3  B: 4\nGrowthFunctionType(int): 1\n  Angle(degrees): 45\n"
                 "GrowthFunctionType(int): 3\n")
    assert e == [("Sec", []), ("A(x)", ["1", "2", "3"]), ("B", ["4"]), ("GrowthFunctionType(int)", ["1"]),
                 ("Angle(degrees)", ["45"]), ("GrowthFunctionType(int)", ["3"])]


def test_setup_matches_what_the_reference_recorded():
    st, z = _load()
    t = st.tissue
    nu = np.where(st.ecm, 0.0, 0.29)
    np.testing.assert_array_equal(st.ecm, z["ecm"])
    np.testing.assert_allclose(2 * t.mu * (1 + nu), z["young"], rtol=1e-15)
    np.testing.assert_array_equal(t.eta, z["eta"])
    np.testing.assert_array_equal(t.ext_visc, z["ext_visc"])
    np.testing.assert_array_equal(t.fixed, z["fixed"])
    np.testing.assert_array_equal(t.exposed, z["exposed"])
    assert sorted(map(tuple, t.slave_master)) == sorted(map(tuple, z["pairs"]))
    rates, angles = st.growth_at(0.0)
    np.testing.assert_array_equal(np.any(rates != 0, axis=1), z["grown"])
    np.testing.assert_array_equal(rates[z["grown"]], np.tile(z["rates"], (int(z["grown"].sum()), 1)))
    assert (angles[z["grown"]] == float(z["angle"])).all()
    assert not st.growth_at(18000.0)[0].any()  # FinalTime 18000 s
    assert t.dt == 3600.0
    assert set(st.not_modelled) == {"explicit-ECM remodelling", "adhesion", "node collapse"}


def test_unsupported_options_are_refused():
    st, z = _load()
    text = " ".join(str(t) for t in z["modelinput_tokens"]).replace("symmetricInX(bool): 0", "symmetricInX(bool): 1")
    with pytest.raises(NotImplementedError, match="symmetry"):
        MI.setup(MI.parse(text), (z["x"], z["place"], z["ttype"], z["circ"], z["conn"], z["xref"]))


def test_loaded_input_gives_the_recorded_first_step_on_the_oracle():
    st, z = _load()
    t = st.tissue.copy()
    t.rates, t.angles = st.growth_at(0.0)
    x, fg, its, norms = O.simulate_dense(t, n_steps=1)
    assert np.abs(x - z["x_step1"]).max() <= 1e-8
    assert its[0] == len(z["du_trace"])


@pytest.mark.gpu
def test_loaded_input_gives_the_recorded_first_step_on_the_gpu():
    st, z = _load()
    xs, stats = st.simulate(n_steps=1)
    assert stats[0]["rc"] == 0
    assert np.abs(xs[0] - z["x_step1"]).max() <= 1e-8
    assert stats[0]["newton_iters"] == len(z["du_trace"])


def test_save_frame_writer_reproduces_the_reference_file():
    """Writing the recorded first frame back gives the reference's Save_Frame text byte for byte."""
    from tissueorigami_b200 import mesh

    st, z = _load()
    text = str(z["frame_text"])
    (time_s, x, flags, conn), = mesh.read_save_frame(text, is_text=True)
    assert time_s == 3600.0
    np.testing.assert_array_equal(conn, z["conn"])
    np.testing.assert_array_equal(x, z["x_step1"])
    block = mesh.save_frame_block(time_s, x, flags[:, 0], flags[:, 1], flags[:, 2], conn, z["xref"])
    assert block == text


def test_save_frame_round_trip(tmp_path):
    from tissueorigami_b200 import mesh

    st, z = _load()
    t = st.tissue
    p = tmp_path / "Save_Frame"
    frames = [(3600.0, z["x_step1"]), (7200.0, z["x_step1"] + 1e-3)]
    mesh.write_save_frame(str(p), frames, t)
    back = mesh.read_save_frame(str(p))
    assert [f[0] for f in back] == [3600.0, 7200.0]
    for (tm, x), (tb, xb, flags, conn) in zip(frames, back):
        assert np.abs(xb - x).max() <= 1e-9 * np.abs(x).max()  # 10 significant digits
        np.testing.assert_array_equal(flags[:, 2], t.at_circumference)


def _variant(z, **repl):
    toks = [str(t) for t in z["modelinput_tokens"]]
    for key, vals in repl.items():
        i = toks.index(key)
        toks[i + 1:i + 1 + len(vals)] = vals
    return MI.setup(MI.parse(" ".join(toks)), (z["x"], z["place"], z["ttype"], z["circ"], z["conn"], z["xref"]))


def _tips(z):
    basal = np.nonzero((z["place"] == 0) & (z["ttype"] == 0))[0]
    xs = z["x"][basal, 0]
    return int(basal[np.argmin(xs)]), int(basal[np.argmax(xs)])


def _added(st, base):
    """The (node, dim) fixes the zero-viscosity rule applied, after checking that every other
    newly fixed DoF is a bound slave above one of them (binding fixes the slaves of a fixed master,
    Simulation.cpp:1344-1436, and runs after the rule)."""
    new = {(int(n), int(d)) for n, d in zip(*np.nonzero(st.tissue.fixed != base.tissue.fixed))}
    applied = set(st.zero_viscosity_fixes)
    masters = {(int(m) // 3, int(m) % 3) for _, m in base.tissue.slave_master}
    slave_of = {(int(s_) // 3, int(s_) % 3): (int(m) // 3, int(m) % 3) for s_, m in base.tissue.slave_master}
    for nd in new - applied:
        assert nd in slave_of and slave_of[nd] in applied and slave_of[nd] in masters, nd
    return sorted(a for a in applied if not base.tissue.fixed[a])


def test_zero_external_viscosity_fixes_the_tips_with_y_symmetry():
    """checkForZeroExternalViscosity (Simulation.cpp:4126-4237): with no drag anywhere and y-symmetry
    the ventral tip is fixed in x, y and z and the dorsal tip in z."""
    st0, z = _load()
    st = _variant(z, **{"DiscProperApicalExternalViscosity:": ["0.0"], "DiscProperBasalExternalViscosity:": ["0.0"]})
    assert not st.tissue.ext_visc.any()
    dorsal, ventral = _tips(z)
    expect = sorted({(ventral, 0), (ventral, 1), (ventral, 2), (dorsal, 2)} - {(n, d) for n, d in zip(*np.nonzero(st0.tissue.fixed))})
    assert _added(st, st0) == expect


def test_zero_external_viscosity_fixes_the_tips_without_symmetry():
    st0, z = _load()
    base = _variant(z, **{"symmetricInY(bool):": ["0"]})
    st = _variant(z, **{"symmetricInY(bool):": ["0"], "DiscProperApicalExternalViscosity:": ["0.0"],
                       "DiscProperBasalExternalViscosity:": ["0.0"]})
    dorsal, ventral = _tips(z)
    third = next(k for k in (1, 2, 3) if k not in (dorsal, ventral))
    want = {(ventral, 0), (ventral, 1), (ventral, 2), (dorsal, 1), (dorsal, 2), (third, 2)}
    assert _added(st, base) == sorted(want - {(n, d) for n, d in zip(*np.nonzero(base.tissue.fixed))})
    # a basal surface fix in z already removes the z rigid motion: no z fixes are added then
    st_z = _variant(z, **{"symmetricInY(bool):": ["0"], "DiscProperApicalExternalViscosity:": ["0.0"],
                         "DiscProperBasalExternalViscosity:": ["0.0"], "BasalSurfaceFix(bool-x,y,z):": ["0", "0", "1"]})
    assert all(d != 2 for _, d in MI.fix_zero_external_viscosity(
        st_z.tissue.fixed.copy() * 0, st_z.tissue.ext_visc, z["place"], z["ttype"], z["x"],
        {k: [False, False, k.startswith("BasalSurfaceFix")] for k in (
            "ApicCircumFix(bool-x,y,z)", "BasalCircumFix(bool-x,y,z)", "LinkerApicCircumFix(bool-x,y,z)",
            "ApicSurfaceFix(bool-x,y,z)", "BasalSurfaceFix(bool-x,y,z)")}, False))


def test_zero_drag_rectangle_is_solvable_only_with_the_tip_fixes():
    """Without drag in x and y the small rectangle (basal nodes fixed in z) can translate and spin
    in its plane: the Newton system is singular. The reference's tip fixes make it solvable."""
    from tissueorigami_b200 import mesh

    t = mesh.small_rectangle(nx=8, ny=5)
    t.ext_visc[:] = 0.0
    fixes = {k: [k == "BasalSurfaceFix(bool-x,y,z)" and d == 2 for d in range(3)]
             for k in ("ApicCircumFix(bool-x,y,z)", "BasalCircumFix(bool-x,y,z)", "LinkerApicCircumFix(bool-x,y,z)",
                       "ApicSurfaceFix(bool-x,y,z)", "BasalSurfaceFix(bool-x,y,z)")}
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    K, g = O.assemble_dense(t, t.x, t.x, vs, inv)
    assert np.linalg.matrix_rank(K) < K.shape[0]
    applied = MI.fix_zero_external_viscosity(t.fixed, t.ext_visc, t.node_placement, np.zeros(t.n_nodes, np.int32), t.x,
                                             fixes, False)
    assert sorted(d for _, d in applied) == [0, 1, 1]
    K, g = O.assemble_dense(t, t.x, t.x, vs, inv)
    assert np.linalg.matrix_rank(K) == K.shape[0]
    x, it, norms = O.newton_step_dense(t, t.x, vs, inv)
    assert np.isfinite(x).all() and norms[-1] <= t.newton_tol
