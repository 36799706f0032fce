"""The lumen term (Lumen.cpp) on the device against the oracle, through the C ABI.

The lumen is the cone from the origin over the apical triangles of a small rectangle (the
reference's volume formula sums (1/6) (x3 x x1) . x2 over them), with its ideal volume growing
two-fold a day.

Tolerances (written per test):
  * residual g and the Jacobian (the device's J plus the rank-one term bulk / (36 V0^2) G G^T
    that it applies by a second solve) against the oracle's: 1e-12 relative to the largest entry;
  * node positions after three steps: 1e-9 of the tissue size, equal Newton counts.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import NewtonRaphsonSolver

pytestmark = pytest.mark.gpu

BULK, FOLD = 1.0e5, 2.0


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _tissue():
    t = mesh.small_rectangle(nx=8, ny=6)
    elems = np.nonzero(t.exposed & 1)[0].astype(np.int32)  # apical faces
    return t, elems


def test_lumen_assembly_matches_oracle():
    t, elems = _tissue()
    rng = np.random.default_rng(9)
    un = t.x.copy()
    uk = un + rng.normal(0.0, 0.05, un.shape)
    _, inv, _, _ = O.grow(t, un, t.fg)
    vs = O.viscosity_surfaces(t, uk)
    rowptr, colidx = O.block_pattern(t)
    tri = O.lumen_triangles(t, elems)
    ideal = O.lumen_volume(t, t.x, tri)
    vals_ref, g_ref = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
    J_ref, g_ref = O.add_lumen(t, O.bsr_to_scipy(rowptr, colidx, vals_ref, t.n_nodes), g_ref, uk, tri, BULK, ideal)
    with NewtonRaphsonSolver.from_tissue(t) as s:
        s.set_lumen(elems, BULK, FOLD, t.x)
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        g, vals, rp, ci, rc = s.assemble(uk, un, t.dt)
        vol, v0, G = s.lumen()
    assert rc == capi.TF_OK
    assert v0 == pytest.approx(ideal, rel=1e-14)
    assert vol == pytest.approx(O.lumen_volume(t, uk, tri), rel=1e-13)
    G = G.reshape(-1)
    J = O.bsr_to_scipy(rp, ci, vals, t.n_nodes).toarray() + BULK / (36.0 * v0 * v0) * np.outer(G, G)
    assert _rel(J, J_ref.toarray()) < 1e-12
    assert _rel(g, g_ref) < 1e-12


def test_lumen_steps_match_oracle():
    t, elems = _tissue()
    x_ref, _, it_ref, _ = O.simulate_sparse(t, n_steps=3, lumen=(elems, BULK, FOLD))
    x_free, _, _, _ = O.simulate_sparse(t, n_steps=3)
    assert np.abs(x_ref - x_free).max() > 1e-3  # the lumen moves the tissue
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
        s.set_lumen(elems, BULK, FOLD, t.x)
        x = t.x.copy()
        its = []
        for _ in range(3):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            its.append(st["newton_iters"])
    assert its == it_ref
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_lumen_refuses_slave_master_pairs():
    t, elems = _tissue()
    with NewtonRaphsonSolver.from_tissue(t) as s:
        s.set_lumen(elems, BULK, FOLD, t.x)
        with pytest.raises(capi.TFError):
            s.set_boundary(t.fixed, t.ext_visc, np.array([[3, 3 * 20]], np.int32))
        s.set_lumen(None)
