"""CPU checks of the oracle (the restatement of the reference path) and of the mesh generators.

These run without a GPU. They pin the oracle's internal consistency: the analytic Jacobian
against central finite differences of the residual (the reference's own numerical-Jacobian
debug path, NewtonRaphsonSolver.cpp:856-885 / Simulation.cpp:6275-6350), the dense and the
sparse assembly against each other, the transposed-solve convention, growth bookkeeping, and
quadratic Newton convergence.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import mesh


def _perturbed(t, seed=0, amp=0.05, eta=0.0):
    rng = np.random.default_rng(seed)
    t = t.copy()
    t.eta[:] = eta
    un = t.x.copy()
    uk = un + rng.normal(0, amp, un.shape)
    fg = np.tile(np.diag([1.02, 1.01, 0.99]).reshape(1, 9), (t.n_elems, 1))
    inv = np.linalg.inv(fg.reshape(-1, 3, 3)).reshape(-1, 9)
    return t, uk, un, inv


def test_rectangle_sizes():
    t = mesh.small_rectangle()
    assert (t.n_nodes, t.n_elems) == (400, 342)
    assert int(t.fixed[:, 2].sum()) == 200 and int(t.fixed[:, :2].sum()) == 0


def test_positive_orientation_and_volume():
    t = mesh.small_rectangle()
    inv, det = O.shape_derivatives(t.xref)
    assert (det > 0).all()
    # sum_g w det(dX/dxi) is the prism volume: 342 prisms of 2 um^2 / 2 x 10 um
    vol = (det / 6.0).sum(axis=1)
    np.testing.assert_allclose(vol, 20.0, rtol=1e-13)


@pytest.mark.parametrize("eta", [0.0, 5.0])
def test_jacobian_is_transpose_of_storage(eta):
    """J = dR/du equals K^T of the reference storage: the viscous tangent is written transposed
    (ShapeBase.cpp:3154-3160) and Pardiso solves the transposed system (NR.cpp:716-723)."""
    t, uk, un, inv = _perturbed(mesh.small_rectangle(nx=4, ny=3), eta=eta)
    t.fixed[:] = 0
    vs = O.viscosity_surfaces(t, uk)
    K, g = O.assemble_dense(t, uk, un, vs, inv)
    n, h = g.size, 1e-6
    Jfd = np.zeros((n, n))
    for j in range(n):
        up = uk.reshape(-1).copy(); up[j] += h
        um = uk.reshape(-1).copy(); um[j] -= h
        _, gp = O.assemble_dense(t, up.reshape(-1, 3), un, vs, inv)
        _, gm = O.assemble_dense(t, um.reshape(-1, 3), un, vs, inv)
        Jfd[:, j] = -(gp - gm) / (2 * h)
    scale = np.abs(Jfd).max()
    assert np.abs(K.T - Jfd).max() / scale < 1e-8
    if eta:
        assert np.abs(K - Jfd).max() / scale > 1e-7  # the untransposed storage is not the Jacobian


def test_sparse_and_dense_assembly_agree():
    t, uk, un, inv = _perturbed(mesh.small_rectangle(nx=6, ny=4), eta=3.0)
    vs = O.viscosity_surfaces(t, uk)
    K, g = O.assemble_dense(t, uk, un, vs, inv)
    rowptr, colidx = O.block_pattern(t)
    vals, g2 = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
    J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes).toarray()
    np.testing.assert_allclose(J, K.T, rtol=0, atol=1e-12 * np.abs(K).max())
    np.testing.assert_allclose(g2, g, rtol=0, atol=1e-12 * np.abs(g).max())


def test_fixed_and_slave_master_elimination():
    """calcutateFixedK and calculateBoundKWithSlavesMasterDoF: identity rows/columns, forces
    folded onto masters, slave displacement equal to the master's after the solve."""
    t, uk, un, inv = _perturbed(mesh.small_rectangle(nx=5, ny=4))
    t.slave_master = np.array([[3 * 7 + 0, 3 * 2 + 0], [3 * 7 + 1, 3 * 2 + 1]], np.int32)
    vs = O.viscosity_surfaces(t, uk)
    K, g = O.assemble_dense(t, uk, un, vs, inv)
    fixed_dofs = np.nonzero(t.fixed.reshape(-1))[0]
    for d in fixed_dofs[:5]:
        assert g[d] == 0.0 and K[d, d] == 1.0
        assert np.count_nonzero(K[d]) == 1 and np.count_nonzero(K[:, d]) == 1
    for s, m in t.slave_master:
        assert g[s] == 0.0 and K[s, s] == 1.0 and np.count_nonzero(K[s]) == 1
    du, st = O.solve_transposed(K, g, t.slave_master)
    assert st == 0
    for s, m in t.slave_master:
        assert du[s] == du[m]


def test_newton_quadratic_convergence():
    t = mesh.small_rectangle()
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    vs = O.viscosity_surfaces(t, t.x)
    x, it, norms = O.newton_step_dense(t, t.x, vs, inv, tol=1e-10)
    assert it <= 6 and norms[-1] <= 1e-10
    # quadratic: each norm below ~ the square of the previous (relative to the first)
    for a, b in zip(norms[:-1], norms[1:]):
        assert b < max(10 * (a / norms[0]) ** 2 * norms[0], 1e-9)


def test_growth_uniform_exponential():
    t = mesh.small_rectangle()
    fg = t.fg.copy()
    for _ in range(3):
        fg, inv, det, rot = O.grow(t, t.x, fg)
        assert not rot.any()
    expect = np.diag([np.exp(3 * 60 * 1e-4), np.exp(3 * 60 * 1e-4), 1.0]).reshape(-1)
    np.testing.assert_allclose(fg, np.tile(expect, (t.n_elems, 1)), rtol=1e-14)
    np.testing.assert_allclose(inv.reshape(-1, 3, 3) @ fg.reshape(-1, 3, 3), np.tile(np.eye(3), (t.n_elems, 1, 1)), atol=1e-14)


def test_growth_rotated_increment():
    """An element turned by +10 degrees about z gets its increment rotated
    (ShapeBase.cpp:1914-2041). The reference reads the angle as atan2(R01, R00) = -10 degrees,
    builds Rz(-10), stores its transpose and applies G^T inc G, i.e. it rotates the increment by
    -10 degrees; the oracle keeps that convention."""
    t = mesh.small_rectangle(nx=3, ny=2)
    th = np.deg2rad(10.0)
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    x = t.x @ R.T
    t.rates[:, 1] = 0.0
    fg, inv, det, rot = O.grow(t, x, t.fg)
    assert rot.all()
    g = np.exp(60 * 1e-4)
    expect = R.T @ np.diag([g, 1.0, 1.0]) @ R
    np.testing.assert_allclose(fg[0].reshape(3, 3), expect, atol=1e-14)


def test_viscosity_surfaces_rectangle():
    t = mesh.small_rectangle()
    vs = O.viscosity_surfaces(t, t.x)
    # total exposed area = apical + basal = 2 * 38 * 18
    assert abs(vs.sum() - 2 * 38 * 18) < 1e-9
    assert vs.min() > 0


def test_mesh_roundtrip(tmp_path):
    t = mesh.small_rectangle(nx=4, ny=3)
    p = tmp_path / "t.mesh"
    mesh.write_mesh(t, str(p))
    x, place, ttype, circ, conn, xref = mesh.read_mesh(str(p))
    np.testing.assert_array_equal(conn, t.conn)
    np.testing.assert_allclose(x, t.x)
    np.testing.assert_allclose(xref, t.xref)
    np.testing.assert_array_equal(place, t.node_placement)


def test_wing_disc_shape():
    t = mesh.wing_disc(n_surface_points=2000)
    inv, det = O.shape_derivatives(t.xref)
    assert (det > 0).all()
    assert t.n_nodes == 3 * (t.n_nodes // 3)
    assert 7000 < t.n_elems < 9000  # 2 layers of ~3.9k triangles
    assert int(t.fixed.sum()) > 0


def test_previous_step_solution_is_a_warm_start():
    """The premise of the Newton loop's warm-started solves (tf_params.krylov_warm_start): for
    Newton iteration k of step n, the solution of iteration k of step n - 1 leaves a residual
    ||g - J du_prev|| well below ||g|| on the first iterations (consecutive steps grow the
    tissue by similar increments). Oracle systems of a 40 x 20 slab, steps 2-3."""
    t = mesh.large_slab(nx=40, ny=20)
    x = np.array(t.x, dtype=np.float64, copy=True)
    fg = np.array(t.fg, dtype=np.float64, copy=True)
    rowptr, colidx = O.block_pattern(t)
    prev, ratios = {}, []
    for step in range(3):
        fg, inv, _, _ = O.grow(t, x, fg)
        vs = O.viscosity_surfaces(t, x)
        un = x.reshape(-1, 3).copy()
        uk, cur = un.copy(), {}
        for k in range(20):
            vals, g = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
            J = O.bsr_to_scipy(rowptr, colidx, vals, t.n_nodes)
            du = O.sparse_direct_solve(J, g)
            cur[k] = du
            if k in prev and k < 3:
                ratios.append(np.linalg.norm(g - J @ prev[k]) / np.linalg.norm(g))
            uk = uk + du.reshape(-1, 3)
            if np.linalg.norm(du) <= t.newton_tol:
                break
        prev = cur
        x = uk.reshape(x.shape)
    assert len(ratios) >= 4
    assert max(ratios) < 0.7, ratios
