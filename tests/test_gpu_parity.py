"""GPU parity of the CUDA path against the oracle, through the C ABI.

Tolerances (written per test):
  * element forces / residual g and Jacobian entries: 1e-12 relative to the largest entry;
  * one linear solve (BiCGStab, rtol 1e-13) against the direct solve of the same system:
    1e-8 relative in ||du|| (the systems have condition numbers ~1e5, so a residual of 1e-13
    leaves up to ~1e-8 in du); with one pass of iterative refinement: 1e-12 relative against
    the solution refined in extended precision and against the direct solve;
  * node positions after N implicit steps: 1e-9 of the tissue size (bounding-box diagonal).
"""
import numpy as np
import pytest
import scipy.sparse.linalg as sla

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import NewtonRaphsonSolver

pytestmark = pytest.mark.gpu


def _state(t, seed=0, amp=0.05, eta=0.0):
    rng = np.random.default_rng(seed)
    t = t.copy()
    t.eta[:] = eta
    un = t.x.copy()
    uk = un + rng.normal(0, amp, un.shape)
    fg = np.tile(np.diag([1.02, 1.01, 0.99]).reshape(1, 9), (t.n_elems, 1))
    inv = np.linalg.inv(fg.reshape(-1, 3, 3)).reshape(-1, 9)
    return t, uk, un, inv


def _gpu_system(t, uk, un, inv, vs, **kw):
    with NewtonRaphsonSolver.from_tissue(t, **kw) as s:
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        g, vals, rowptr, colidx, rc = s.assemble(uk, un, t.dt)
    return g, O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes), rc


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("eta", [0.0, 4.0])
@pytest.mark.parametrize("scatter,teams", [(capi.TF_SCATTER_ATOMIC, 16), (capi.TF_SCATTER_COLOURED, 8),
                                           (capi.TF_SCATTER_ATOMIC, 32), (capi.TF_SCATTER_COLOURED, 32),
                                           (capi.TF_SCATTER_STAGED, 8), (capi.TF_SCATTER_STAGED, 16),
                                           (capi.TF_SCATTER_STAGED, 32)])
def test_assembly_matches_oracle(eta, scatter, teams):
    t, uk, un, inv = _state(mesh.small_rectangle(nx=9, ny=6), eta=eta)
    vs = O.viscosity_surfaces(t, uk)
    rowptr, colidx = O.block_pattern(t)
    vals, g_ref = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
    J_ref = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).toarray()
    g, J, rc = _gpu_system(t, uk, un, inv, vs, scatter=scatter, elems_per_block=teams)
    assert rc == capi.TF_OK
    assert _rel(J.toarray(), J_ref) < 1e-12
    assert _rel(g, g_ref) < 1e-12


def test_assembly_disc_matches_oracle():
    t, uk, un, inv = _state(mesh.wing_disc(n_surface_points=800), amp=0.02)
    vs = O.viscosity_surfaces(t, uk)
    rowptr, colidx = O.block_pattern(t)
    vals, g_ref = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
    J_ref = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes)
    g, J, rc = _gpu_system(t, uk, un, inv, vs)
    assert rc == capi.TF_OK
    assert abs(J - J_ref).max() / abs(J_ref).max() < 1e-12
    assert _rel(g, g_ref) < 1e-12


def test_slave_master_assembly_matches_dense_oracle():
    """calculateBoundKWithSlavesMasterDoF on the fixed pattern: routed scatter == N^T K N + I."""
    t, uk, un, inv = _state(mesh.small_rectangle(nx=6, ny=4), eta=2.0)
    # bind x,y of two apical nodes to other apical nodes (both directions untouched by fixing)
    t.slave_master = np.array([[3 * 9 + 0, 3 * 3 + 0], [3 * 9 + 1, 3 * 3 + 1], [3 * 21 + 0, 3 * 15 + 0]], np.int32)
    vs = O.viscosity_surfaces(t, uk)
    K, g_ref = O.assemble_dense(t, uk, un, vs, inv)
    g, J, rc = _gpu_system(t, uk, un, inv, vs)
    assert rc == capi.TF_OK
    assert _rel(J.toarray(), K.T) < 1e-12
    assert _rel(g, g_ref) < 1e-12


@pytest.mark.parametrize("persistent", [0, 1])
def test_solve_matches_direct(persistent):
    """Both solve paths (graph-replayed iteration kernels, persistent cooperative kernel) against
    SuperLU: 1e-8 relative in ||du||, fixed DoFs exactly zero."""
    t = mesh.small_disc(7, 1500, 1200.0)
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx)
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc()
    du_ref = sla.spsolve(J, g)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, persistent=persistent) as s:
        rp, ci = s.pattern()
        np.testing.assert_array_equal(rp, rowptr)
        np.testing.assert_array_equal(ci, colidx)
        du, rc, iters, rr = s.solveForDeltaU(vals, g)
    assert rc == capi.TF_OK and rr <= 1e-13
    assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8
    fixed = t.fixed.reshape(-1) != 0
    assert np.all(du[fixed] == 0.0)


def _exact_solution(J, g, passes=4):
    """The FP64-rounded solution of J x = g: SuperLU followed by refinement passes whose residual
    is summed in extended precision (long double), so the result is limited by rounding only."""
    J = J.tocsr()
    lu = sla.splu(J.tocsc())
    x = lu.solve(g)
    for _ in range(passes):
        prod = J.data.astype(np.longdouble) * x.astype(np.longdouble)[J.indices]
        r = g.astype(np.longdouble) - np.add.reduceat(prod, J.indptr[:-1])
        x = np.asarray(x.astype(np.longdouble) + lu.solve(np.asarray(r, np.float64)).astype(np.longdouble), np.float64)
    return x


@pytest.mark.parametrize("persistent", [0, 1])
def test_refined_solve_matches_exact_solution_to_1e12(persistent):
    """solveForDeltaU to 1e-12 relative. BiCGStab alone stops at ||g - J du|| <= rtol ||g||,
    which leaves an error up to kappa(J) x rtol in du (kappa_1 ~ 6e4 here, so up to ~1e-8 at
    rtol 1e-13: the 1e-8 gate of test_solve_matches_direct). One pass of iterative refinement
    (FP64 residual, a second solve for the correction; Pardiso refines once too) brings du to
    the rounding level, the accuracy of the direct solve itself: both are compared with the
    solution refined in extended precision, and with each other, at 1e-12."""
    t = mesh.small_disc(7, 1500, 1200.0)
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx)
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes)
    x_star = _exact_solution(J, g)
    du_lu = sla.spsolve(J.tocsc(), g)
    assert np.linalg.norm(du_lu - x_star) / np.linalg.norm(x_star) < 1e-12
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, krylov_refine=2, persistent=persistent) as s:
        du, rc, iters, rr = s.solveForDeltaU(vals, g)
    assert rc == capi.TF_OK and rr <= 1e-13
    assert np.linalg.norm(du - x_star) / np.linalg.norm(x_star) < 1e-12
    assert np.linalg.norm(du - du_lu) / np.linalg.norm(du_lu) < 1e-12
    fixed = t.fixed.reshape(-1) != 0
    assert np.all(du[fixed] == 0.0)


def test_newton_step_matches_oracle_small_rectangle():
    t = mesh.small_rectangle()
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    x_ref, it_ref, norms_ref = O.newton_step_dense(t, t.x, vs, inv, tol=t.newton_tol)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        x, rc, st = s.updateStepNR(t.x, t.dt)
    assert rc == capi.TF_OK
    assert st["newton_iters"] == it_ref
    np.testing.assert_allclose(st["du_norm"][0], norms_ref[0], rtol=1e-9)
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_ten_time_steps_small_rectangle():
    """Small rectangle, 10 implicit steps of 60 s, Newton tolerance 1e-10 (growth prologue on the
    device): positions within 1e-9 of the tissue size of the oracle's dense-LU run."""
    t = mesh.small_rectangle()
    x_ref, fg_ref, it_ref, _ = O.simulate_dense(t, n_steps=10)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
        x = t.x.copy()
        its = []
        for _ in range(10):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            its.append(st["newton_iters"])
        fg, _ = s.get_growth()
    assert its == it_ref
    np.testing.assert_allclose(fg, fg_ref, rtol=1e-13, atol=1e-15)
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_warm_started_solves_match_cold_ones():
    """tf_params.krylov_warm_start: from the second step on, each Newton iteration's conjugate
    gradients start from the previous step's solution of the same iteration, with the same
    stopping rule. Four steps of the disc: the same Newton counts and positions as cold-started
    solves within 1e-9 of the tissue size, both against the oracle's sparse steps, and fewer
    Krylov iterations over the warm steps."""
    t = mesh.wing_disc(n_surface_points=1500)
    res = {}
    for warm in (0, 1):
        with NewtonRaphsonSolver.from_tissue(t, krylov_warm_start=warm) as s:
            x = t.x.copy()
            its, kry = [], 0
            for k in range(4):
                x, rc, st = s.runOneStep(x, t.dt)
                assert rc == capi.TF_OK, (warm, k)
                its.append(st["newton_iters"])
                if k > 0:
                    kry += st["krylov_iters_total"]
        res[warm] = (x, its, kry)
    assert res[0][1] == res[1][1]
    assert np.abs(res[0][0] - res[1][0]).max() <= 1e-9 * t.size
    assert res[1][2] < res[0][2], (res[1][2], res[0][2])
    fg = np.array(t.fg, dtype=np.float64, copy=True)
    x_o = np.array(t.x, dtype=np.float64, copy=True)
    for k in range(4):
        fg, inv, _, _ = O.grow(t, x_o, fg)
        vs = O.viscosity_surfaces(t, x_o)
        x_o, it_o, _ = O.newton_step_sparse(t, x_o, vs, inv)
        assert it_o == res[1][1][k], (k, it_o, res[1][1])
    assert np.abs(res[1][0] - x_o.reshape(res[1][0].shape)).max() <= 1e-9 * t.size


@pytest.mark.parametrize("persistent", [0, 1])
def test_time_steps_disc_matches_sparse_oracle(persistent):
    t = mesh.small_disc(11, 3000, 2000.0, n_steps=3)
    x_ref, fg_ref, it_ref, _ = O.simulate_sparse(t, n_steps=3)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14, persistent=persistent) as s:
        x = t.x.copy()
        for _ in range(3):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


@pytest.mark.parametrize("precond", ["two_level", "block_jacobi"])
def test_column_smoother_solve_matches_direct(precond):
    """Block-Jacobi over a prism column's three nodes (9x9 blocks; the wing disc numbers each
    column's nodes consecutively) against SuperLU and against 3x3 node blocks: 1e-8 relative in
    ||du||, no more BiCGStab iterations than with node blocks."""
    pc = {"two_level": capi.TF_PRECOND_TWO_LEVEL, "block_jacobi": capi.TF_PRECOND_BLOCK_JACOBI}[precond]
    t = mesh.wing_disc(n_surface_points=3000)
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx)
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc()
    du_ref = sla.spsolve(J, g)
    iters = {}
    for sn in (0, 1):
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=pc, smoother_nodes=sn) as s:
            assert s.smoother_block() == (3 if sn == 0 else 1)
            du, rc, iters[sn], rr = s.solveForDeltaU(vals, g)
        assert rc == capi.TF_OK and rr <= 1e-13
        assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8
        assert np.all(du[t.fixed.reshape(-1) != 0] == 0.0)
    assert iters[0] <= iters[1]


def test_column_smoother_steps_match_sparse_oracle():
    """Implicit steps of a three-surface disc with the default (column) smoother: positions
    within 1e-9 of the tissue size of the sparse oracle, the same Newton iteration counts."""
    t = mesh.wing_disc(n_surface_points=1500, n_steps=2)
    x_ref, fg_ref, it_ref, _ = O.simulate_sparse(t, n_steps=2)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
        assert s.smoother_block() == 3
        x = t.x.copy()
        its = []
        for _ in range(2):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            its.append(st["newton_iters"])
    assert its == list(it_ref)
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


@pytest.mark.parametrize("nodes", [2, 4])
def test_forced_smoother_blocks_solve_matches_direct(nodes):
    """Blocks of G consecutive nodes that are not columns (forced G = 2 and the largest, G = 4,
    on a one-layer rectangle of 108 nodes) still precondition the same system: 1e-8 relative in
    ||du|| against SuperLU."""
    t = mesh.small_rectangle(nx=9, ny=6)
    t, uk, un, inv = _state(t)
    vs = O.viscosity_surfaces(t, uk)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
    du_ref = sla.spsolve(O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc(), g)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, smoother_nodes=nodes) as s:
        assert s.smoother_block() == nodes
        du, rc, iters, rr = s.solveForDeltaU(vals, g)
    assert rc == capi.TF_OK and rr <= 1e-13
    assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8


def test_smoother_nodes_argument_checks():
    t = mesh.small_disc(7, 600, 1200.0)  # two surfaces: columns of two nodes
    with NewtonRaphsonSolver.from_tissue(t) as s:
        assert s.smoother_block() == 2
    with NewtonRaphsonSolver.from_tissue(t, persistent=0) as s:
        assert s.smoother_block() == 1  # the chunked path keeps node blocks
    with pytest.raises(capi.TFError):
        NewtonRaphsonSolver.from_tissue(t, smoother_nodes=5)


def test_status_newton_cap():
    t = mesh.small_rectangle(nx=5, ny=4)
    with NewtonRaphsonSolver.from_tissue(t, max_newton_iters=0) as s:
        x, rc, st = s.runOneStep(t.x, t.dt)
    assert rc == capi.TF_NEWTON_NOT_CONVERGED and st["newton_iters"] == 1


def test_status_krylov_cap():
    t = mesh.small_rectangle(nx=5, ny=4)
    with NewtonRaphsonSolver.from_tissue(t, krylov_max_iters=1, max_newton_iters=1) as s:
        x, rc, st = s.runOneStep(t.x, t.dt)
    assert rc in (capi.TF_KRYLOV_MAX_ITERS, capi.TF_NEWTON_NOT_CONVERGED)
    assert st["krylov_iters_max"] <= 1


def test_status_nonfinite_input():
    t = mesh.small_rectangle(nx=5, ny=4)
    x = t.x.copy()
    x[3, 0] = np.nan
    with NewtonRaphsonSolver.from_tissue(t) as s:
        x2, rc, st = s.updateStepNR(x, t.dt)
    assert rc == capi.TF_NONFINITE


def test_status_inverted_element():
    t = mesh.small_rectangle(nx=5, ny=4)
    x = t.x.copy()
    apical = np.nonzero(t.node_placement == mesh.APICAL)[0]
    x[apical, 2] = -5.0  # push the apical surface below the basal one
    with NewtonRaphsonSolver.from_tissue(t, max_newton_iters=1) as s:
        g = np.zeros(3)
        g, vals, rp, ci, rc = s.assemble(x, t.x, t.dt)
    assert rc == capi.TF_ELEMENT_INVERTED


def test_schedule_and_autotune():
    t = mesh.wing_disc(n_surface_points=800)
    with NewtonRaphsonSolver.from_tissue(t) as s:
        sch = s.schedule()
        assert sch["n_colours"] > 0
        tuned = s.autotune(t.x, t.dt)
        assert tuned["scatter"] in (capi.TF_SCATTER_ATOMIC, capi.TF_SCATTER_COLOURED, capi.TF_SCATTER_STAGED)
        assert tuned["elems_per_block"] in (8, 16, 32)
        me, ms = s.time_kernels(5)
        assert me > 0 and ms > 0


def test_direct_solve_matches_scipy_and_krylov():
    """tf_solve_direct (cuSOLVER sparse Cholesky / QR) against SuperLU and against BiCGStab."""
    t = mesh.small_disc(7, 1500, 1200.0)
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx)
    du_ref = sla.spsolve(O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc(), g)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13) as s:
        du_d, rc_d, ms, method = s.solve_direct(vals, g)
        du_k, rc_k, _, _ = s.solveForDeltaU(vals, g)
    assert rc_d == capi.TF_OK and method in (1, 2) and ms > 0
    assert np.linalg.norm(du_d - du_ref) / np.linalg.norm(du_ref) < 1e-10
    assert np.linalg.norm(du_k - du_d) / np.linalg.norm(du_d) < 1e-8


def test_ilu0_solve_matches_direct_with_fewer_iterations():
    """Multicolour block ILU(0)-preconditioned BiCGStab: same solution as SuperLU (1e-8 relative),
    and no more iterations than the block-Jacobi preconditioner needs."""
    t = mesh.small_disc(7, 1500, 1200.0)
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx)
    du_ref = sla.spsolve(O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc(), g)
    iters = {}
    for pc in (capi.TF_PRECOND_BLOCK_JACOBI, capi.TF_PRECOND_ILU0):
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=pc, persistent=0) as s:
            du, rc, it, rr = s.solveForDeltaU(vals, g)
        assert rc == capi.TF_OK and rr <= 1e-13
        assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8
        iters[pc] = it
    assert iters[capi.TF_PRECOND_ILU0] <= iters[capi.TF_PRECOND_BLOCK_JACOBI]


def test_ilu0_time_steps_match_oracle():
    """Three implicit steps of a small disc with the ILU(0) preconditioner: positions within 1e-9
    of the tissue size of the oracle's sparse-LU run."""
    t = mesh.small_disc(11, 3000, 2000.0, n_steps=3)
    x_ref, fg_ref, it_ref, _ = O.simulate_sparse(t, n_steps=3)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14, precond=capi.TF_PRECOND_ILU0) as s:
        x = t.x.copy()
        for _ in range(3):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_two_level_solve_matches_direct_with_fewer_iterations():
    """Block-Jacobi + aggregation coarse correction (rigid-body modes on node-range aggregates):
    the SuperLU solution to 1e-8, fixed DoFs exactly zero, fewer BiCGStab iterations than
    block-Jacobi alone."""
    t = mesh.wing_disc(n_surface_points=1500)
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx)
    du_ref = sla.spsolve(O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc(), g)
    fixed = t.fixed.reshape(-1) != 0
    iters = {}
    for pc in (capi.TF_PRECOND_BLOCK_JACOBI, capi.TF_PRECOND_TWO_LEVEL):
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=pc) as s:
            du, rc, it, rr = s.solveForDeltaU(vals, g)
            pc_eff, n_coarse, refreshes = s.preconditioner()
        assert pc_eff == pc
        if pc == capi.TF_PRECOND_TWO_LEVEL:
            assert n_coarse > 0 and refreshes == 1
        assert rc == capi.TF_OK and rr <= 1e-13
        assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8
        assert np.all(du[fixed] == 0.0)
        iters[pc] = it
    assert iters[capi.TF_PRECOND_TWO_LEVEL] < iters[capi.TF_PRECOND_BLOCK_JACOBI]


def test_two_level_time_steps_match_oracle():
    t = mesh.small_disc(11, 3000, 2000.0, n_steps=3)
    x_ref, fg_ref, it_ref, _ = O.simulate_sparse(t, n_steps=3)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14, precond=capi.TF_PRECOND_TWO_LEVEL) as s:
        x = t.x.copy()
        for _ in range(3):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_two_level_with_slaves_matches_block_jacobi():
    """Slave DoFs are left out of the coarse modes: with slave-master pairs the two-level
    solve gives the block-Jacobi positions (1e-9 of the tissue size) after two steps."""
    t = mesh.small_rectangle(nx=12, ny=8)
    t.slave_master = np.array([[3 * 30 + 0, 3 * 20 + 0], [3 * 30 + 1, 3 * 20 + 1], [3 * 41 + 2, 3 * 33 + 2]], np.int32)
    out = {}
    for pc in (capi.TF_PRECOND_BLOCK_JACOBI, capi.TF_PRECOND_TWO_LEVEL):
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14, precond=pc) as s:
            x = t.x.copy()
            for _ in range(2):
                x, rc, st = s.runOneStep(x, t.dt)
                assert rc == capi.TF_OK
        out[pc] = x
    assert np.abs(out[capi.TF_PRECOND_TWO_LEVEL] - out[capi.TF_PRECOND_BLOCK_JACOBI]).max() <= 1e-9 * t.size
    # the slaves follow their masters exactly
    x = out[capi.TF_PRECOND_TWO_LEVEL].reshape(-1)
    for s_, m_ in t.slave_master:
        assert x[s_] - t.x.reshape(-1)[s_] == pytest.approx(x[m_] - t.x.reshape(-1)[m_], abs=1e-12 * t.size)


@pytest.mark.parametrize("degrees", [10.0, -25.0, 0.5])
def test_device_growth_rotation_branch_matches_oracle(degrees):
    """The growth prologue's rotation test (ShapeBase::CalculateGrowthRotationByF,
    ShapeBase.cpp:1914-2041): elements turned about z by more than the 0.017 (about 1 degree)
    threshold get their growth increment rotated back into the reference frame, those turned
    less do not. The tissue is turned rigidly with every DoF fixed, so the step's mechanics leave
    it where it is; the device's Fg after the step must equal the oracle's at 1e-12, with the
    branch taken exactly where the oracle takes it."""
    t = mesh.small_rectangle(nx=6, ny=4)
    t.fixed[:] = 1
    t.rates[:, 0], t.rates[:, 1] = 3e-4, 0.5e-4  # anisotropic, so the rotation changes Fg
    th = np.deg2rad(degrees)
    R = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]])
    x = t.x @ R.T
    fg_ref, _, _, rot = O.grow(t, x, t.fg)
    assert rot.all() == (abs(degrees) > 1.0) and rot.any() == (abs(degrees) > 1.0)
    with NewtonRaphsonSolver.from_tissue(t) as s:
        x_out, rc, _ = s.runOneStep(x, t.dt)
        assert rc == capi.TF_OK
        fg, _ = s.get_growth()
    np.testing.assert_array_equal(x_out, x)
    assert np.abs(fg.reshape(-1, 9) - fg_ref).max() / np.abs(fg_ref).max() <= 1e-12


def test_host_newton_loop_over_newton_iteration_matches_device_loop():
    """The reference's updateStepNR loop kept on the host (checkConvergenceViaDeltaU,
    updateUkInIteration), each iteration's assembly and solve through tf_newton_iteration: the
    same positions and iteration count as the device loop of tf_newton_step and the oracle."""
    t = mesh.small_rectangle()
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    x_ref, it_ref, _ = O.newton_step_dense(t, t.x, vs, inv, tol=t.newton_tol)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        x_dev, rc, st = s.updateStepNR(t.x, t.dt)
        assert rc == capi.TF_OK
        un = t.x.reshape(-1).copy()
        uk = un.copy()
        k, converged = 0, False
        while not converged:
            du, rc, _, _ = s.newton_iteration(uk, un, t.dt)
            assert rc == capi.TF_OK
            converged = not (np.linalg.norm(du) > t.newton_tol)
            uk = uk + du
            k += 1
            assert k <= 21
    assert k == st["newton_iters"] == it_ref
    assert np.abs(uk.reshape(-1, 3) - x_dev).max() <= 1e-12 * t.size
    assert np.abs(uk.reshape(-1, 3) - x_ref).max() <= 1e-9 * t.size


def test_external_force_enters_the_residual_on_free_dofs():
    """NewtonRaphsonSolver::addExernalForces: gSum += gExt, then the fixed DoFs are zeroed."""
    t, uk, un, inv = _state(mesh.small_rectangle(nx=7, ny=5))
    vs = O.viscosity_surfaces(t, uk)
    f = np.random.default_rng(2).normal(0.0, 50.0, (t.n_nodes, 3))
    with NewtonRaphsonSolver.from_tissue(t) as s:
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        g0, J0, _, _, rc0 = s.assemble(uk, un, t.dt)
        s.set_external_force(f)
        g1, J1, _, _, rc1 = s.assemble(uk, un, t.dt)
        s.set_external_force(None)
        g2, _, _, _, _ = s.assemble(uk, un, t.dt)
    assert rc0 == rc1 == capi.TF_OK
    want = np.where(t.fixed.reshape(-1) != 0, 0.0, f.reshape(-1))
    assert np.abs((g1 - g0) - want).max() <= 1e-12 * np.abs(g0).max()
    assert _rel(J1, J0) <= 1e-14  # the Jacobian does not see the force (atomic sums may reorder)
    assert np.abs(g2 - g0).max() <= 1e-12 * np.abs(g0).max()


def _disc_system():
    t = mesh.small_disc(7, 1500, 1200.0)
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, t.x, t.x, vs, inv, rowptr, colidx)
    return t, rowptr, colidx, vals, g


@pytest.mark.parametrize("precond", [capi.TF_PRECOND_BLOCK_JACOBI, capi.TF_PRECOND_TWO_LEVEL])
@pytest.mark.parametrize("smoother", [1, 2])
def test_conjugate_gradients_match_direct_and_bicgstab(precond, smoother):
    """The persistent solve by conjugate gradients (the default for a symmetric J: no internal
    viscosity) against SuperLU (1e-8, as BiCGStab) and against BiCGStab on the same system, for
    node and column smoother blocks, with and without the coarse correction."""
    t, rowptr, colidx, vals, g = _disc_system()
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc()
    du_ref = sla.spsolve(J, g)
    out = {}
    for method in (capi.TF_KRYLOV_CG, capi.TF_KRYLOV_BICGSTAB):
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=precond, smoother_nodes=smoother,
                                             krylov_method=method) as s:
            du, rc, iters, rr = s.solveForDeltaU(vals, g)
            assert rc == capi.TF_OK and rr <= 1e-13
            assert s.krylov_method() == {capi.TF_KRYLOV_CG: 2, capi.TF_KRYLOV_BICGSTAB: 1}[method]
        out[method] = du
        assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8
        assert np.all(du[t.fixed.reshape(-1) != 0] == 0.0)
    assert np.linalg.norm(out[capi.TF_KRYLOV_CG] - out[capi.TF_KRYLOV_BICGSTAB]) / np.linalg.norm(du_ref) < 1e-8


def test_conjugate_gradients_fall_back_to_bicgstab_on_an_indefinite_system():
    """A symmetric but indefinite system (one node's diagonal block negated): the preconditioned
    residual of CG has (r, M^-1 r) < 0 when the right-hand side sits on that node, CG stops with a
    non-positive curvature and the library solves the system again with BiCGStab."""
    t, rowptr, colidx, vals, g = _disc_system()
    free = np.nonzero(t.fixed.sum(axis=1) == 0)[0]
    node = int(free[len(free) // 2])
    k = int(np.nonzero(colidx[rowptr[node]:rowptr[node + 1]] == node)[0][0]) + rowptr[node]
    vals = vals.copy()
    vals[k] = -vals[k]
    g = np.zeros_like(g)
    g[3 * node:3 * node + 3] = [1.0, -2.0, 0.5]
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).tocsc()
    du_ref = sla.spsolve(J, g)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=capi.TF_PRECOND_BLOCK_JACOBI,
                                         krylov_method=capi.TF_KRYLOV_CG) as s:
        du, rc, iters, rr = s.solveForDeltaU(vals, g)
        assert s.krylov_method() == 3
    assert rc == capi.TF_OK and rr <= 1e-13
    assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8


@pytest.mark.parametrize("method", [capi.TF_KRYLOV_CG, capi.TF_KRYLOV_BICGSTAB])
def test_ten_time_steps_small_rectangle_either_krylov_method(method):
    """Ten steps of the small rectangle with either Krylov method, against the dense oracle. The
    first Newton Jacobian of every step has one negative eigenvalue (about -1.9 against a largest
    of 5.3e4: the rigid in-plane rotation, which only the drag resists, under the compressive
    prestress of the fresh growth increment), so conjugate gradients may meet a non-positive
    curvature there and hand the solve to BiCGStab (method 3); the later iterations are positive
    definite."""
    t = mesh.small_rectangle()
    x_ref, _, it_ref, _ = O.simulate_dense(t, n_steps=10)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14, krylov_method=method) as s:
        x = t.x.copy()
        its = []
        for _ in range(10):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            assert st["krylov_method"] in {capi.TF_KRYLOV_CG: (2, 3), capi.TF_KRYLOV_BICGSTAB: (1,)}[method]
            its.append(st["newton_iters"])
    assert its == it_ref
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size
