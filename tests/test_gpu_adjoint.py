"""GPU tests of the discrete adjoint of the growth time loop (tf_adjoint_forward/backward).

A growth map parameterised by a bilinear grid drives a small clamped disc for a few implicit
steps; the loss is the squared node-position misfit to a target shape made by a hidden grid.
The adjoint gradient (through a torch.autograd.Function that lives in this test harness only)
is checked against central finite differences (h = 1e-6 on the grid values) of the GPU forward
path and of the oracle, to 1e-5 relative to the largest gradient entry.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import NewtonRaphsonSolver

pytestmark = pytest.mark.gpu

N_STEPS, CHECKPOINT, GRID, RATE = 4, 2, 4, 1e-4


def _setup():
    t = mesh.small_disc(21, 400, 1500.0, n_steps=N_STEPS)
    t.newton_tol = 1e-13
    idx, w = mesh.bilinear_growth_weights(t, GRID)
    W = np.zeros((t.n_elems, GRID * GRID))
    for k in range(4):
        np.add.at(W, (np.arange(t.n_elems), idx[:, k]), w[:, k])
    return t, W


def _rates(W, p):
    r = RATE * (W @ p)
    out = np.zeros((W.shape[0], 3))
    out[:, 0] = r
    out[:, 1] = r
    return out


class GrowthForward(torch.autograd.Function):
    """rates [E,3] -> final positions [N,3] through the GPU time loop; backward = the adjoint."""

    @staticmethod
    def forward(ctx, rates, solver, t):
        solver.set_growth(t.fg, rates.detach().numpy(), t.angles)
        x, rc, st = solver.adjoint_forward(t.x, N_STEPS, t.dt, CHECKPOINT)
        assert rc == capi.TF_OK
        ctx.solver = solver
        return torch.from_numpy(x)

    @staticmethod
    def backward(ctx, grad_x):
        dr, _, rc, st = ctx.solver.adjoint_backward(grad_x.numpy())
        assert rc == capi.TF_OK
        return torch.from_numpy(dr), None, None


def _gpu_loss(s, t, W, p, target):
    s.set_growth(t.fg, _rates(W, p), t.angles)
    x, rc, _ = s.adjoint_forward(t.x, N_STEPS, t.dt, CHECKPOINT)
    assert rc == capi.TF_OK
    return float(((x - target) ** 2).sum())


def _oracle_loss(t, W, p, target):
    tt = t.copy()
    tt.rates = _rates(W, p)
    x, _, _, _ = O.simulate_dense(tt, n_steps=N_STEPS, tol=1e-13)
    return float(((x - target) ** 2).sum())


def test_adjoint_gradient_matches_finite_differences():
    t, W = _setup()
    rng = np.random.default_rng(7)
    p_hidden = rng.uniform(0.5, 1.5, GRID * GRID)
    p = rng.uniform(0.5, 1.5, GRID * GRID)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
        s.set_growth(t.fg, _rates(W, p_hidden), t.angles)
        target, rc, _ = s.adjoint_forward(t.x, N_STEPS, t.dt, CHECKPOINT)
        assert rc == capi.TF_OK
        pt = torch.tensor(p, requires_grad=True)
        Wt = torch.from_numpy(W)
        r = RATE * (Wt @ pt)
        rates = torch.stack([r, r, torch.zeros_like(r)], dim=1)
        x = GrowthForward.apply(rates, s, t)
        loss = ((x - torch.from_numpy(target)) ** 2).sum()
        loss.backward()
        grad = pt.grad.numpy()
        scale = np.abs(grad).max()
        assert scale > 0
        h = 1e-6
        for k in rng.choice(GRID * GRID, 4, replace=False):
            e = np.zeros_like(p)
            e[k] = h
            fd = (_gpu_loss(s, t, W, p + e, target) - _gpu_loss(s, t, W, p - e, target)) / (2 * h)
            assert abs(fd - grad[k]) <= 1e-5 * scale, (k, fd, grad[k])
        # the reference path (oracle, dense LU) for two parameters
        for k in rng.choice(GRID * GRID, 2, replace=False):
            e = np.zeros_like(p)
            e[k] = h
            fd = (_oracle_loss(t, W, p + e, target) - _oracle_loss(t, W, p - e, target)) / (2 * h)
            assert abs(fd - grad[k]) <= 1e-5 * scale, (k, fd, grad[k])


def test_adjoint_forward_matches_time_steps():
    t, W = _setup()
    p = np.full(GRID * GRID, 1.0)
    with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
        s.set_growth(t.fg, _rates(W, p), t.angles)
        xa, rc, _ = s.adjoint_forward(t.x, N_STEPS, t.dt, CHECKPOINT)
        s.set_growth(t.fg, _rates(W, p), t.angles)
        x = t.x.copy()
        for _ in range(N_STEPS):
            x, rc, _ = s.runOneStep(x, t.dt)
    assert np.abs(xa - x).max() <= 1e-12 * t.size
