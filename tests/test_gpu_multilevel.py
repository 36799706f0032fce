"""The multilevel coarse space of a single tissue (TF_PRECOND_MULTILEVEL), through the C ABI.

Tolerances (written per test):
  * one linear solve (rtol 1e-13) against the SuperLU solution of the same system: 1e-8 relative
    in ||du|| (condition numbers ~1e5), fixed DoFs exactly zero;
  * node positions after N implicit steps: 1e-9 of the tissue size against the sparse oracle;
  * the full large slab: one time step with the multilevel space against the same step with
    block-Jacobi alone (two independent preconditioners of the same Newton iteration), 1e-9 of
    the tissue size, the same Newton iteration count.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import NewtonRaphsonSolver

pytestmark = pytest.mark.gpu


def _system(t):
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx, threads=16)
    return vals, g, rowptr, colidx


@pytest.mark.parametrize("method", [capi.TF_KRYLOV_AUTO, capi.TF_KRYLOV_BICGSTAB])
def test_multilevel_solve_matches_direct_with_fewer_iterations(method):
    """A 200 x 100-point slab (80,000 nodes: 1,024 leaves, levels of 1,024 / 256 / 64 sets): the
    SuperLU solution to 1e-8 with under half the iterations block-Jacobi needs."""
    t = mesh.large_slab(nx=200, ny=100)
    vals, g, rowptr, colidx = _system(t)
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes)
    du_ref = O.sparse_direct_solve(J, g, O.nested_dissection(t, rowptr, colidx))
    fixed = t.fixed.reshape(-1) != 0
    iters = {}
    for pc in (capi.TF_PRECOND_BLOCK_JACOBI, capi.TF_PRECOND_MULTILEVEL):
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=pc, krylov_method=method) as s:
            du, rc, it, rr = s.solveForDeltaU(vals, g)
            pc_eff, n_coarse, refreshes = s.preconditioner()
        assert pc_eff == pc
        if pc == capi.TF_PRECOND_MULTILEVEL:
            assert n_coarse == 6 * (1024 + 256 + 64) and refreshes == 1
        assert rc == capi.TF_OK and rr <= 1e-13
        assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8
        assert np.all(du[fixed] == 0.0)
        iters[pc] = it
    assert 2 * iters[capi.TF_PRECOND_MULTILEVEL] < iters[capi.TF_PRECOND_BLOCK_JACOBI], iters


def test_multilevel_disc_solve_matches_direct():
    """The wing disc's three-node columns with the column smoother (G = 3) inside the leaves."""
    t = mesh.wing_disc(n_surface_points=4000)
    vals, g, rowptr, colidx = _system(t)
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes)
    du_ref = O.sparse_direct_solve(J, g, O.nested_dissection(t, rowptr, colidx))
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=capi.TF_PRECOND_MULTILEVEL) as s:
        du, rc, it, rr = s.solveForDeltaU(vals, g)
        pc_eff, n_coarse, _ = s.preconditioner()
        assert s.smoother_block() == 3
    assert pc_eff == capi.TF_PRECOND_MULTILEVEL and n_coarse > 0
    assert rc == capi.TF_OK and rr <= 1e-13
    assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8


def test_multilevel_time_steps_match_oracle():
    t = mesh.small_disc(11, 3000, 2000.0, n_steps=3)
    x_ref, _, it_ref, _ = O.simulate_sparse(t, n_steps=3)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14, precond=capi.TF_PRECOND_MULTILEVEL) as s:
        x = t.x.copy()
        its = []
        for _ in range(3):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            its.append(st["newton_iters"])
        assert s.preconditioner()[0] == capi.TF_PRECOND_MULTILEVEL
    assert its == it_ref
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_multilevel_with_slaves_matches_block_jacobi():
    """Slave DoFs are left out of every set's modes: the block-Jacobi positions after two steps."""
    t = mesh.small_rectangle(nx=24, ny=16)
    t.slave_master = np.array([[3 * 30 + 0, 3 * 20 + 0], [3 * 30 + 1, 3 * 20 + 1], [3 * 41 + 2, 3 * 33 + 2]], np.int32)
    out = {}
    for pc in (capi.TF_PRECOND_BLOCK_JACOBI, capi.TF_PRECOND_MULTILEVEL):
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14, precond=pc) as s:
            x = t.x.copy()
            for _ in range(2):
                x, rc, st = s.runOneStep(x, t.dt)
                assert rc == capi.TF_OK
        out[pc] = x
    assert np.abs(out[capi.TF_PRECOND_MULTILEVEL] - out[capi.TF_PRECOND_BLOCK_JACOBI]).max() <= 1e-9 * t.size


def test_large_slab_step_multilevel_matches_block_jacobi():
    """The full large slab (2,000,000 nodes): the default preconditioner takes the multilevel space
    (32,768 leaves, five levels); one time step matches the block-Jacobi step."""
    t = mesh.large_slab()
    out, its = {}, {}
    for pc in (capi.TF_PRECOND_TWO_LEVEL, capi.TF_PRECOND_BLOCK_JACOBI):
        with NewtonRaphsonSolver.from_tissue(t, precond=pc) as s:
            x, rc, st = s.runOneStep(t.x.copy(), t.dt)
            assert rc == capi.TF_OK
            if pc == capi.TF_PRECOND_TWO_LEVEL:
                pc_eff, n_coarse, _ = s.preconditioner()
                assert pc_eff == capi.TF_PRECOND_MULTILEVEL
                assert n_coarse == 6 * (32768 + 8192 + 2048 + 512 + 128)
        out[pc], its[pc] = x, st["newton_iters"]
    assert its[capi.TF_PRECOND_TWO_LEVEL] == its[capi.TF_PRECOND_BLOCK_JACOBI]
    assert np.abs(out[capi.TF_PRECOND_TWO_LEVEL] - out[capi.TF_PRECOND_BLOCK_JACOBI]).max() <= 1e-9 * t.size
