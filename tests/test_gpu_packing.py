"""Packing (node-node contact) on the device against the oracle, through the C ABI.

The stacked-sheet tissue puts the apical surfaces of two one-layer rectangles 0.5 um apart, so
every apical node of the lower sheet away from the box's upper edges has a packing partner.

Tolerances (written per test):
  * pairs and their order: equal; packingThreshold and node masses: 1e-13 relative;
  * residual g and Jacobian (element pattern + the pairs' blocks): 1e-12 relative to the largest entry;
  * node positions after three steps: 1e-9 of the tissue size, equal Newton counts and pair counts.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import NewtonRaphsonSolver

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_detection_matches_oracle():
    t = mesh.stacked_sheets()
    pairs_ref, thr_ref = O.detect_packing(t, t.x)
    assert len(pairs_ref) == 45
    with NewtonRaphsonSolver.from_tissue(t, packing=True) as s:
        n = s.detect_packing(t.x)
        pairs, thr, mass, _ = s.packing()
    assert n == len(pairs_ref)
    np.testing.assert_array_equal(pairs, pairs_ref)
    assert abs(thr - thr_ref) <= 1e-13 * thr_ref
    assert _rel(mass, O.node_masses(t, t.fg)) <= 1e-13


def test_assembly_with_packing_matches_oracle():
    t = mesh.stacked_sheets()
    rng = np.random.default_rng(5)
    un = t.x.copy()
    uk = un + rng.normal(0.0, 0.05, un.shape)
    _, inv, _, _ = O.grow(t, un, t.fg)
    vs = O.viscosity_surfaces(t, uk)
    rowptr, colidx = O.block_pattern(t)
    pairs_ref, thr = O.detect_packing(t, un)
    mass = O.node_masses(t, t.fg)
    vals_ref, g_ref = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
    J_ref, g_ref = O.add_packing(t, O.bsr_to_scipy(rowptr, colidx, vals_ref, t.n_nodes), g_ref, uk, pairs_ref, mass, thr)
    with NewtonRaphsonSolver.from_tissue(t, packing=True) as s:
        s.detect_packing(un)
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        g, vals, rp, ci, rc = s.assemble(uk, un, t.dt)
        pairs, _, _, dfdx = s.packing()
    assert rc == capi.TF_OK
    np.testing.assert_array_equal(pairs, pairs_ref)
    # the pairs' blocks outside the element pattern, as the device applies them
    free = t.fixed.reshape(-1) == 0
    rows, cols, v = [], [], []
    for p, (i, j) in enumerate(pairs):
        for a, b in ((i, j), (j, i)):
            for r in range(3):
                for c in range(3):
                    if free[3 * a + r] and free[3 * b + c]:
                        rows.append(3 * a + r)
                        cols.append(3 * b + c)
                        v.append(dfdx[p, r, c])
    n = 3 * t.n_nodes
    J = O.bsr_to_scipy(rp, ci, vals, t.n_nodes) + sp.csr_matrix((v, (rows, cols)), shape=(n, n))
    assert _rel(J.toarray(), J_ref.toarray()) < 1e-12
    assert _rel(g, g_ref) < 1e-12


def test_steps_with_packing_match_oracle():
    t = mesh.stacked_sheets()
    counts_ref = []
    x_ref, _, it_ref, _ = O.simulate_sparse(t, n_steps=3, packing=True, pair_counts=counts_ref)
    assert counts_ref == [45, 15, 45]
    with NewtonRaphsonSolver.from_tissue(t, packing=True) as s:
        x = t.x.copy()
        its, counts = [], []
        for _ in range(3):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            # the pairs' repulsion makes J indefinite (91 of 720 eigenvalues negative at the first
            # iterate): MINRES with the |D| block preconditioner solves those systems
            assert st["krylov_method"] == 4
            its.append(st["newton_iters"])
            counts.append(len(s.packing()[0]))
    assert counts == counts_ref
    assert its == it_ref
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_packing_moves_the_sheets_apart():
    """Without packing the same three steps end 0.26 um away: the contact terms are not inert."""
    t = mesh.stacked_sheets()
    out = {}
    for pk in (False, True):
        with NewtonRaphsonSolver.from_tissue(t, packing=pk) as s:
            x = t.x.copy()
            for _ in range(3):
                x, rc, _ = s.runOneStep(x, t.dt)
                assert rc == capi.TF_OK
        out[pk] = x
    assert np.abs(out[True] - out[False]).max() > 0.1


def test_packing_refuses_what_it_does_not_support():
    t = mesh.stacked_sheets()
    with NewtonRaphsonSolver.from_tissue(t, packing=True) as s:
        assert s.detect_packing(t.x) == 45
        # slave-master pairs with packing
        with pytest.raises(capi.TFError):
            s.set_boundary(t.fixed, t.ext_visc, np.array([[3, 3 * 20]], np.int32))
        # a direct solve while the step has pairs
        vals = np.zeros((s.pattern()[1].shape[0], 9))
        with pytest.raises(capi.TFError):
            s.solve_direct(vals, np.zeros(3 * t.n_nodes))
        s.set_packing(None)
        assert s.packing()[0].shape[0] == 0


@pytest.mark.parametrize("name", ["wing_disc", "large_slab"])
def test_device_detection_finds_no_pairs_in_the_benchmark_tissues(name):
    """The device's detector agrees with the oracle's on the benchmark tissues: no pair at the
    start (the oracle's full-run assertions are in test_gpu_full_size.py)."""
    t = getattr(mesh, name)()
    with NewtonRaphsonSolver.from_tissue(t, packing=True) as s:
        assert s.detect_packing(t.x) == 0
        _, thr, mass, _ = s.packing()
    _, thr_ref = O.detect_packing(t, t.x)
    # the threshold averages up to 6 M side lengths: the oracle sums them in order, the device
    # with atomics; the order alone moves such a sum by up to ~n eps (2.7e-11 measured on the slab)
    assert abs(thr - thr_ref) <= 1e-9 * thr_ref
    assert _rel(mass, O.node_masses(t, t.fg)) <= 1e-12
