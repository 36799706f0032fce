"""GPU parity at the full sizes of the benchmark workloads.

The smaller parity tests (test_gpu_parity.py, test_gpu_batch.py, test_gpu_adjoint.py) check the
CUDA path against the oracle on miniatures. These tests run the workloads the benchmark times, at
their full sizes, through the C ABI:

* wing disc (79,650 prisms, 60,441 nodes): the whole assembly against the oracle's faithful element
  loop, 1e-12 relative to the largest entry; two full time steps against the oracle's sparse
  Newton step (SuperLU standing in for Pardiso): the same Newton iteration counts and positions
  within 1e-9 of the tissue size;
* large slab (2,991,006 prisms, 2,000,000 nodes): the full assembly on the GPU; the rows of 4,000
  randomly drawn nodes against the oracle's assembly of every prism that touches them (a row of J
  and of g depends only on the prisms around its node), 1e-12 relative for J; for g, 1e-12
  relative or twice the oracle's own rounding floor at these coordinates, whichever is larger
  (the slab spans 500 um at 0.5 um spacing, so the deformation gradient is a difference of terms
  ~1000 times larger than itself: the oracle's g moves by ~2.5e-12 relative under a rigid
  translation of all coordinates, while the order of its sums moves it by ~2e-16);
* batch of 256 uneven tissues (1.34 M prisms): positions and Newton counts of every tissue after
  three steps against separate single-tissue runs, 1e-9 of each tissue's size;
* adjoint fit (wing disc, 32 x 32 bilinear growth grid, 20 steps, checkpoint every 5): the adjoint
  gradient against central finite differences (h = 1e-6) of the GPU forward run on 32 random
  parameters, 1e-5 relative to the largest gradient entry. The oracle's finite differences at this
  size would take hours (one forward run is 80 SuperLU factorisations of 180k unknowns); the
  oracle's gradient check runs on the small disc of test_gpu_adjoint.py;
* packing: the reference adds contact forces for node pairs that come closer than 0.4 x the
  local element side (Simulation::detectPacingNodes); the path here computes the step without them,
  so each workload must stay free of such pairs. The oracle's detector runs on the positions at the
  start of every step of C1 (10 steps), C2 (50), C4 (30, all 256 tissues), on C3 (20 steps) at the
  start of every fifth step, and on every final state, and finds no pair.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import BatchSolver, NewtonRaphsonSolver

pytestmark = pytest.mark.gpu


def _rel_rows(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_wing_disc_full_assembly_matches_oracle():
    t = mesh.wing_disc()
    assert t.n_elems == 79650 and t.n_nodes == 60441
    rng = np.random.default_rng(11)
    un = t.x.copy()
    uk = un + rng.normal(0.0, 0.02, un.shape)
    _, inv, _, _ = O.grow(t, un, t.fg)
    vs = O.viscosity_surfaces(t, uk)
    rowptr, colidx = O.block_pattern(t)
    vals_ref, g_ref = O.assemble_bsr(t, uk, un, vs, inv, rowptr, colidx)
    with NewtonRaphsonSolver.from_tissue(t) as s:
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        g, vals, rp, ci, rc = s.assemble(uk, un, t.dt)
    assert rc == capi.TF_OK
    np.testing.assert_array_equal(rp, rowptr)
    np.testing.assert_array_equal(ci, colidx)
    assert _rel_rows(vals, vals_ref) < 1e-12
    assert _rel_rows(g, g_ref) < 1e-12


def test_wing_disc_two_full_steps_match_oracle():
    t = mesh.wing_disc()
    n_steps = 2
    x_ref, _, it_ref, tr_ref = O.simulate_sparse(t, n_steps=n_steps, reorder=True)
    with NewtonRaphsonSolver.from_tissue(t) as s:
        x = t.x.copy()
        its = []
        for _ in range(n_steps):
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            its.append(st["newton_iters"])
    assert its == it_ref
    assert np.abs(x - x_ref).max() <= 1e-9 * t.size


def test_large_slab_assembly_matches_oracle_on_sampled_rows():
    t = mesh.large_slab()
    assert t.n_elems == 2991006 and t.n_nodes == 2000000
    rng = np.random.default_rng(12)
    un = t.x.copy()
    uk = un + rng.normal(0.0, 0.01, un.shape)
    _, inv, _, _ = O.grow(t, un, t.fg)
    vs = O.viscosity_surfaces(t, uk)
    with NewtonRaphsonSolver.from_tissue(t) as s:
        s.set_inv_fg(inv)
        s.set_viscosity_surface(vs)
        g, vals, rowptr, colidx, rc = s.assemble(uk, un, t.dt)
    assert rc == capi.TF_OK
    rows = np.sort(rng.choice(t.n_nodes, 4000, replace=False))
    touch = np.isin(t.conn, rows).any(axis=1)
    sub = t.copy()
    sub.conn, sub.xref = t.conn[touch], t.xref[touch]
    sub.lam, sub.mu, sub.eta = t.lam[touch], t.mu[touch], t.eta[touch]
    vals_ref, g_ref = O.assemble_bsr(sub, uk, un, vs, inv[touch], rowptr, colidx, threads=16)
    blocks = np.concatenate([np.arange(rowptr[r], rowptr[r + 1]) for r in rows])
    dofs = (3 * rows[:, None] + np.arange(3)[None, :]).ravel()
    assert _rel_rows(vals[blocks], vals_ref[blocks]) < 1e-12
    # the oracle's rounding floor: its g under a rigid translation of every coordinate
    c = -0.5 * (t.x.min(axis=0) + t.x.max(axis=0))
    shifted = _translated(sub, c)
    _, g_shift = O.assemble_bsr(shifted, uk + c, un + c, vs, inv[touch], rowptr, colidx, threads=16)
    floor = _rel_rows(g_shift[dofs], g_ref[dofs])
    assert _rel_rows(g[dofs], g_ref[dofs]) < max(1e-12, 2.0 * floor), floor


def _translated(t, c):
    out = t.copy()
    out.x = t.x + c
    out.xref = t.xref + np.tile(c, 6)[None, :]
    return out


def test_batch_of_256_matches_sequential_runs():
    ts = mesh.batch_tissues(n_tissues=256)
    n_steps = 3
    with BatchSolver(ts) as b:
        x = b.join([t.x for t in ts])
        its_batch = []
        for _ in range(n_steps):
            x, rc, _ = b.runOneStep(x, ts[0].dt)
            assert rc == capi.TF_OK
            its_batch.append(b.tissue_stats()["newton_iters"].copy())
        xs = b.split(x)
    its_batch = np.array(its_batch).T
    for i, t in enumerate(ts):
        with NewtonRaphsonSolver.from_tissue(t) as s:
            xx = t.x.copy()
            for k in range(n_steps):
                xx, rc, st = s.runOneStep(xx, t.dt)
                assert rc == capi.TF_OK
                assert st["newton_iters"] == its_batch[i, k], (i, k)
        assert np.abs(xs[i] - xx).max() <= 1e-9 * t.size, i


def _adjoint_problem():
    t = mesh.wing_disc()
    grid, n_steps, k = 32, 20, 5
    idx, w = mesh.bilinear_growth_weights(t, grid)
    rng = np.random.default_rng(1004)
    gx, gy = np.meshgrid(np.linspace(t.x[:, 0].min(), t.x[:, 0].max(), grid),
                         np.linspace(t.x[:, 1].min(), t.x[:, 1].max(), grid), indexing="xy")
    hidden = 2e-4 * np.exp(-(gx ** 2 + gy ** 2).ravel() / (2 * 40.0 ** 2)) * (1 + rng.uniform(-0.1, 0.1, grid * grid))
    theta = hidden * (1 + rng.uniform(-0.2, 0.2, grid * grid))

    def rates(p):
        r = (w * p[idx]).sum(axis=1)
        out = np.zeros((t.n_elems, 3))
        out[:, 0] = r
        out[:, 1] = r
        return out

    return t, idx, w, hidden, theta, rates, n_steps, k


def test_adjoint_gradient_matches_finite_differences_full_size():
    t, idx, w, hidden, theta, rates, n_steps, k = _adjoint_problem()
    with NewtonRaphsonSolver.from_tissue(t) as s:
        s.set_growth(t.fg, rates(hidden), t.angles)
        target, rc, _ = s.adjoint_forward(t.x, n_steps, t.dt, k)
        assert rc == capi.TF_OK

        def loss(p):
            s.set_growth(t.fg, rates(p), t.angles)
            xf, rc_, _ = s.adjoint_forward(t.x, n_steps, t.dt, k)
            assert rc_ == capi.TF_OK
            return float(np.sum((xf - target) ** 2)), xf

        _, xf = loss(theta)
        dr, _, rcb, _ = s.adjoint_backward(2.0 * (xf - target))
        assert rcb == capi.TF_OK
        grad = np.zeros(theta.shape[0])
        np.add.at(grad, idx.ravel(), (w * (dr[:, 0] + dr[:, 1])[:, None]).ravel())
        support = np.flatnonzero(np.bincount(idx.ravel(), weights=w.ravel(), minlength=theta.shape[0]) > 0)
        pick = np.random.default_rng(32).choice(support, 32, replace=False)
        h = 1e-6
        fd = []
        for p in pick:
            e = np.zeros_like(theta)
            e[p] = h
            fd.append((loss(theta + e)[0] - loss(theta - e)[0]) / (2 * h))
    fd = np.array(fd)
    scale = np.abs(grad).max()
    assert scale > 0
    err = np.abs(fd - grad[pick]).max() / scale
    assert err < 1e-5, err


def _assert_no_pairs(t, x, where):
    pairs, _ = O.detect_packing(t, x)
    assert pairs.shape[0] == 0, (where, pairs[:5])


@pytest.mark.parametrize("name", ["small_rectangle", "wing_disc", "large_slab"])
def test_single_tissue_workloads_stay_free_of_packing(name):
    t = {"small_rectangle": mesh.small_rectangle, "wing_disc": mesh.wing_disc, "large_slab": mesh.large_slab}[name]()
    every = 5 if name == "large_slab" else 1
    with NewtonRaphsonSolver.from_tissue(t) as s:
        x = t.x.copy()
        for k in range(t.n_steps):
            if k % every == 0:
                _assert_no_pairs(t, x, (name, k))
            x, rc, _ = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK, (name, k)
    _assert_no_pairs(t, x, (name, t.n_steps))


def test_batch_workload_stays_free_of_packing():
    ts = mesh.batch_tissues(n_tissues=256)
    with BatchSolver(ts) as b:
        x = b.join([t.x for t in ts])
        for k in range(ts[0].n_steps):
            for i, (t, xi) in enumerate(zip(ts, b.split(x))):
                _assert_no_pairs(t, xi, ("batch", i, k))
            x, rc, _ = b.runOneStep(x, ts[0].dt)
            assert rc == capi.TF_OK, k
        for i, (t, xi) in enumerate(zip(ts, b.split(x))):
            _assert_no_pairs(t, xi, ("batch", i, ts[0].n_steps))
