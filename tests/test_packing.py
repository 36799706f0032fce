"""Node-node packing detection (Simulation::detectPacingNodes, Simulation.cpp:7997-8153).

The reference runs packing detection at the start of every time step and, for the pairs it
finds, adds implicit contact forces and Jacobian terms to the Newton system. The CUDA path of
this repository computes the step without those terms, so it equals the reference's step exactly
when the detection finds no pair. These CPU tests pin the oracle's detector (a cell-list search)
to a literal restatement of the reference's all-pairs loop, on meshes with and without pairs.
tests/test_gpu_full_size.py then asserts that every benchmark configuration stays free of pairs
over its full number of steps.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import mesh


def _literal_detect(t, x):
    """The reference's loops, line for line (getAverageSideLength :3197-3262, detectPacingNodes
    :8001-8070), in plain Python: only for small meshes."""
    bb0 = [100000.0, 100000.0]
    bb1 = [-100000.0, -100000.0]
    for n in range(t.n_nodes):
        for d in range(2):
            if x[n, d] < bb0[d]:
                bb0[d] = x[n, d]
            elif x[n, d] > bb1[d]:
                bb1[d] = x[n, d]
    size = [bb1[0] - bb0[0], bb1[1] - bb0[1]]
    grid = [[0.0] * 5 for _ in range(10)]
    cnt = [[0.0] * 5 for _ in range(10)]

    def avg(c, pairs):
        s, k = 0.0, 0
        for a, b in pairs:
            d2 = float(np.sum((x[c[a]] - x[c[b]]) ** 2))
            if d2 > 0:
                s += d2 ** 0.5
                k += 1
        return s / k if k else 0.0

    for e in range(t.n_elems):
        if t.peripodial[e]:
            continue
        c = t.conn[e]
        cur = avg(c, [(3, 4), (3, 5), (4, 5)])
        if t.exposed[e] & 2:
            cur = avg(c, [(0, 1), (0, 2), (1, 2)])
        cen = x[c].mean(axis=0)
        rx = math.floor((cen[0] - bb0[0]) / size[0])
        ry = math.floor(((cen[1] - bb0[1]) / size[1]) / 2.0)
        rx = min(9, max(0, rx))
        ry = min(4, max(0, ry))
        grid[rx][ry] += cur
        cnt[rx][ry] += 1
    gsq = [[0.0] * 5 for _ in range(10)]
    for i in range(10):
        for j in range(5):
            if cnt[i][j] > 0:
                grid[i][j] /= cnt[i][j]
            grid[i][j] *= 0.4
            gsq[i][j] = grid[i][j] * grid[i][j]
    neig = [set() for _ in range(t.n_nodes)]
    for c in t.conn:
        for a in c:
            neig[a].update(int(b) for b in c if b != a)
    pairs = []
    for i in range(t.n_nodes):
        if t.node_placement[i] not in (0, 1):
            continue
        gx = math.floor((x[i, 0] - bb0[0]) / size[0])
        gy = math.floor((x[i, 1] - bb0[1]) / size[1])
        t2 = gsq[gx][gy]
        for j in range(i + 1, t.n_nodes):
            if t.node_placement[j] not in (0, 1) or t.node_placement[j] != t.node_placement[i]:
                continue
            if j in neig[i]:
                continue
            if float(np.sum((x[i] - x[j]) ** 2)) < t2:
                pairs.append((i, j))
    return np.array(pairs, np.int32).reshape(-1, 2)


def _two_rectangles(gap, nx=6, ny=4):
    """Two single-layer rectangles side by side in x, `gap` um apart (one mesh)."""
    a = mesh.small_rectangle(nx=nx, ny=ny)
    b = mesh.small_rectangle(nx=nx, ny=ny)
    shift = (nx - 1) * 2.0 + gap
    t = a.copy()
    n = a.n_nodes
    t.x = np.concatenate([a.x, b.x + [shift, 0.0, 0.0]])
    t.conn = np.concatenate([a.conn, b.conn + n]).astype(np.int32)
    t.xref = t.x[t.conn].reshape(-1, 18)
    for f in ("lam", "mu", "eta", "exposed", "peripodial", "angles"):
        setattr(t, f, np.concatenate([getattr(a, f), getattr(b, f)]))
    for f in ("fixed", "ext_visc", "node_placement", "at_circumference"):
        setattr(t, f, np.concatenate([getattr(a, f), getattr(b, f)]))
    t.rates = np.concatenate([a.rates, b.rates])
    t.fg = np.concatenate([a.fg, b.fg])
    return t


def test_small_rectangle_has_no_packing_pairs():
    t = mesh.small_rectangle()
    pairs, thr = O.detect_packing(t, t.x)
    assert pairs.shape == (0, 2)
    # packingThreshold = 0.4 x the columnar average side length (2, 2 and 2 sqrt 2 um sides)
    assert abs(thr - 0.4 * (4.0 + 2.0 * math.sqrt(2.0)) / 3.0) < 1e-12


def test_facing_edges_of_two_rectangles_pack():
    gap = 0.5  # below 0.4 x the 2.28 um average side length
    t = _two_rectangles(gap)
    pairs, _ = O.detect_packing(t, t.x)
    ref = _literal_detect(t, t.x)
    np.testing.assert_array_equal(pairs, ref)
    # every facing node of the same surface and row packs with its partner across the gap, except
    # the top row: the reference picks a node's threshold cell as floor((pos - box min) / box
    # size) (Simulation.cpp:8042-8044), which is 1 on the box's upper edge, and that cell of the
    # 10 x 5 grid holds no element (elements land in cell 0: floor of a relative position < 1),
    # so its threshold is 0
    assert pairs.shape[0] == 3 * 2
    d = np.linalg.norm(t.x[pairs[:, 0]] - t.x[pairs[:, 1]], axis=1)
    np.testing.assert_allclose(d, gap)
    assert (t.node_placement[pairs[:, 0]] == t.node_placement[pairs[:, 1]]).all()


def test_detector_matches_literal_loops_on_perturbed_meshes():
    rng = np.random.default_rng(7)
    for gap in (0.3, 0.8, 1.2):
        t = _two_rectangles(gap, nx=7, ny=5)
        x = t.x + rng.normal(0.0, 0.25, t.x.shape)
        np.testing.assert_array_equal(O.detect_packing(t, x)[0], _literal_detect(t, x))
    t = mesh.small_disc(3, 300, 1000.0)
    x = t.x + rng.normal(0.0, 0.6, t.x.shape)
    pairs = O.detect_packing(t, x)[0]
    np.testing.assert_array_equal(pairs, _literal_detect(t, x))


def test_packing_jacobian_matches_finite_differences_of_the_forces():
    """The oracle's calculatePackingJacobian3D restatement is the derivative of its
    calculatePackingForcesImplicit3D restatement (central differences, h = 1e-6, 1e-7 relative)."""
    t = mesh.stacked_sheets()
    fg, _, _, _ = O.grow(t, t.x, t.fg)
    pairs, thr = O.detect_packing(t, t.x)
    assert len(pairs) == 45
    mass = O.node_masses(t, fg)
    rng = np.random.default_rng(3)
    x = t.x + rng.normal(0.0, 0.05, t.x.shape)
    _, D = O.packing_terms(t, x, pairs, mass, thr)
    h = 1e-6
    for p in (0, 17, 44):
        i, j = pairs[p]
        num = np.zeros((3, 3))
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, c] += h
            xm[i, c] -= h
            fp, _ = O.packing_terms(t, xp, pairs[p:p + 1], mass, thr)
            fm, _ = O.packing_terms(t, xm, pairs[p:p + 1], mass, thr)
            num[:, c] = (fp[i] - fm[i]) / (2 * h)
        assert np.abs(num - D[p]).max() <= 1e-7 * np.abs(D[p]).max()
        assert np.allclose(D[p], D[p].T, rtol=0, atol=1e-12 * np.abs(D[p]).max())


def test_node_masses_sum_to_the_grown_volume():
    """Each prism hands det(Fg) x its volume to its six nodes: the masses sum to the grown volume
    of both sheets (2 x 18 x 10 x 4 um^3 times det(Fg))."""
    t = mesh.stacked_sheets()
    fg, _, _, _ = O.grow(t, t.x, t.fg)
    mass = O.node_masses(t, fg)
    det = np.linalg.det(fg.reshape(-1, 3, 3))
    assert np.allclose(det, det[0])
    assert mass.sum() == pytest.approx(2 * 18.0 * 10.0 * 4.0 * det[0], rel=1e-13)


def test_lumen_jacobian_is_the_derivative_of_the_lumen_forces():
    """The oracle's restatement of Lumen::calculateJacobian (with the rank-one term) is minus the
    derivative of its Lumen::calculateResiduals forces and symmetric (central differences,
    h = 1e-6, 1e-7 relative)."""
    t = mesh.small_rectangle(nx=6, ny=4)
    tri = O.lumen_triangles(t, np.nonzero(t.exposed & 1)[0])
    rng = np.random.default_rng(1)
    x = t.x + rng.normal(0, 0.1, t.x.shape)
    ideal = 0.97 * O.lumen_volume(t, t.x, tri)
    _, K = O.lumen_terms(t, x, tri, 1000.0, ideal)
    n = 3 * t.n_nodes
    free = t.fixed.reshape(-1) == 0
    h = 1e-6
    J = np.zeros((n, n))
    for c in range(n):
        xp, xm = x.copy().reshape(-1), x.copy().reshape(-1)
        xp[c] += h
        xm[c] -= h
        fp, _ = O.lumen_terms(t, xp.reshape(-1, 3), tri, 1000.0, ideal)
        fm, _ = O.lumen_terms(t, xm.reshape(-1, 3), tri, 1000.0, ideal)
        J[:, c] = -(fp.reshape(-1) - fm.reshape(-1)) / (2 * h)
    J *= np.outer(free, free)
    assert np.abs(K - J).max() <= 1e-7 * np.abs(J).max()
    assert np.abs(K - K.T).max() <= 1e-14 * np.abs(K).max()
