"""GPU test of tf_solve_bsr_noalloc, the allocation-free variant of the linear solve.

Some host applications give all device memory to their own allocator, or to a pool fixed at
start-up, and cannot let a library call cudaMalloc / cudaFree per solve. For them the library
offers tf_solve_bsr_noalloc: the caller passes device buffers it owns (here allocated by torch,
standing in for the caller's allocator) and the solve keeps its scratch in a fixed array inside
the library. The test calls it twice in a row on two different systems and checks each answer
against tf_solve (the allocating entry point) on the same system, within the 1e-8 relative
tolerance the solve parity tests use. It also checks that a system larger than the fixed
scratch is refused with TF_ERR_TOO_LARGE.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import NewtonRaphsonSolver

pytestmark = pytest.mark.gpu


def _system(t, x, inv_fg):
    vs = O.viscosity_surfaces(t, x)
    rowptr, colidx = O.block_pattern(t)
    vals, g = O.assemble_bsr(t, x, t.x, vs, inv_fg, rowptr, colidx)
    return rowptr, colidx, vals, g


def _noalloc(L, n_nodes, rowptr, colidx, vals, g):
    import torch

    dev = torch.device("cuda:0")
    rp = torch.from_numpy(rowptr).to(dev)
    ci = torch.from_numpy(colidx).to(dev)
    va = torch.from_numpy(np.ascontiguousarray(vals.reshape(-1))).to(dev)
    gg = torch.from_numpy(np.ascontiguousarray(g)).to(dev)
    du = torch.full_like(gg, float("nan"))
    torch.cuda.synchronize()
    it = ctypes.c_int32()
    rr = ctypes.c_double()
    rc = L.tf_solve_bsr_noalloc(n_nodes, rp.data_ptr(), ci.data_ptr(), va.data_ptr(), gg.data_ptr(), du.data_ptr(),
                                1e-13, 20000, None, ctypes.byref(it), ctypes.byref(rr))
    return rc, du.cpu().numpy(), it.value, rr.value


def test_noalloc_solve_matches_tf_solve_on_two_calls():
    L = capi.load()
    t = mesh.small_disc(7, 1500, 1200.0)
    assert t.n_nodes <= capi.TF_NOALLOC_MAX_NODES
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    rng = np.random.default_rng(5)
    x2 = t.x + rng.normal(0.0, 0.02, t.x.shape)
    systems = [_system(t, t.x, inv), _system(t, x2, inv)]
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13) as s:
        refs = [s.solveForDeltaU(vals, g) for (_, _, vals, g) in systems]
    for (rowptr, colidx, vals, g), (du_ref, rc_ref, _, _) in zip(systems, refs):
        assert rc_ref == capi.TF_OK
        rc, du, iters, rr = _noalloc(L, t.n_nodes, rowptr, colidx, vals, g)
        assert rc == capi.TF_OK, capi.STATUS_NAMES.get(rc, rc)
        assert iters > 0 and rr <= 1e-13
        assert np.all(np.isfinite(du))
        assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8


def test_noalloc_rejects_systems_beyond_its_scratch():
    L = capi.load()
    rc = L.tf_solve_bsr_noalloc(capi.TF_NOALLOC_MAX_NODES + 1, 16, 16, 16, 16, 16, 1e-12, 10, None, None, None)
    assert rc == capi.TF_ERR_TOO_LARGE


def test_noalloc_solve_at_its_maximum_size():
    """A system of exactly TF_NOALLOC_MAX_NODES block rows (a 128 x 64-node rectangle, two node
    surfaces, rim clamped) fills every region of the fixed scratch - work vectors, block-Jacobi
    inverses, diagonal slots and the reduction partials of the widest launch. Two calls in a row
    on two systems against tf_solve, 1e-8 relative."""
    L = capi.load()
    t = mesh.small_rectangle(nx=128, ny=64)
    t.fixed[t.at_circumference != 0, :] = 1
    assert t.n_nodes == capi.TF_NOALLOC_MAX_NODES
    fg, inv, _, _ = O.grow(t, t.x, t.fg)
    rng = np.random.default_rng(9)
    x2 = t.x + rng.normal(0.0, 0.01, t.x.shape)
    systems = [_system(t, t.x, inv), _system(t, x2, inv)]
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-13, precond=capi.TF_PRECOND_BLOCK_JACOBI) as s:
        refs = [s.solveForDeltaU(vals, g) for (_, _, vals, g) in systems]
    for (rowptr, colidx, vals, g), (du_ref, rc_ref, _, _) in zip(systems, refs):
        assert rc_ref == capi.TF_OK
        rc, du, iters, rr = _noalloc(L, t.n_nodes, rowptr, colidx, vals, g)
        assert rc == capi.TF_OK, capi.STATUS_NAMES.get(rc, rc)
        assert iters > 0 and rr <= 1e-13
        assert np.linalg.norm(du - du_ref) / np.linalg.norm(du_ref) < 1e-8
