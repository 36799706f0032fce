"""Growth prologue pinned against the reference's own output.

tests/golden/run07008_growth.npz comes from the reference's no-Pardiso regression run 07008
(made by tests/golden/make_run07008_growth.py): a wing-disc mesh grown uniformly (0.2 / 0.1 per
hour along DV / AP at 45 degrees, columnar layer only, from 0 to 18000 s) for 11 steps of
3600 s with the mechanics left unsolved, so node positions never move. The golden file holds
every element's growth tensor Fg after every step.

Both the oracle's restatement of the growth prologue (CPU) and the library's device prologue
(GPU, through the C ABI, with every DoF fixed so that the Newton step leaves the positions
where they are) must reproduce it. Tolerance: 1e-12 relative to the largest entry (the
reference's exp and GSL products against ours, compounded over five increments).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "run07008_growth.npz")
TOL = 1e-12


def _tissue():
    z = np.load(GOLDEN)
    E = z["conn"].shape[0]
    grown = z["grown"]
    rates = np.zeros((E, 3))
    rates[grown] = z["rates"]
    lam, mu = mesh.lame(np.full(E, 100.0), 0.29)
    N = z["x"].shape[0]
    t = mesh.Tissue("run07008", z["conn"].astype(np.int32), z["xref"], z["x"], lam, mu, np.zeros(E),
                    np.ones((N, 3), np.uint8), np.zeros((N, 3)), np.zeros(E, np.uint8), np.zeros(E, np.uint8),
                    rates, np.full(E, float(z["angle"])), z["place"].astype(np.int32), z["circ"].astype(np.int32),
                    dt=float(z["dt"]), n_steps=z["frames"].shape[0], newton_tol=1e-8)
    return t, z


def _active(z, step):
    """Growth applies at simulation time t = step * dt when InitialTime <= t < FinalTime."""
    t = step * float(z["dt"])
    return float(z["t0"]) <= t < float(z["t1"])


def _check(fg, golden, step):
    err = np.abs(fg - golden).max() / np.abs(golden).max()
    assert err <= TOL, f"step {step}: Fg differs from the reference by {err:.2e} (relative)"


def test_fixture_is_what_the_reference_says():
    t, z = _tissue()
    frames = z["frames"]
    assert frames.shape == (11, 138, 9) and int(z["grown"].sum()) == 46
    # growth stops after five steps (FinalTime 18000 s)
    np.testing.assert_array_equal(frames[5], frames[10])
    assert not np.array_equal(frames[3], frames[4])


def test_oracle_growth_matches_reference_output():
    t, z = _tissue()
    fg = t.fg.copy()
    zero = t.copy()
    zero.rates = np.zeros_like(t.rates)
    for step in range(z["frames"].shape[0]):
        fg, inv, det, rot = O.grow(t if _active(z, step) else zero, t.x, fg)
        assert not rot.any()  # the tissue never moves, so no growth rotation is triggered
        _check(fg, z["frames"][step], step)


@pytest.mark.gpu
def test_device_growth_matches_reference_output():
    from tissueorigami_b200 import capi
    from tissueorigami_b200.newton import NewtonRaphsonSolver

    t, z = _tissue()
    with NewtonRaphsonSolver.from_tissue(t) as s:
        x = t.x.copy()
        for step in range(z["frames"].shape[0]):
            if step > 0 and _active(z, step - 1) and not _active(z, step):
                fg_now, _ = s.get_growth()
                s.set_growth(fg_now, np.zeros_like(t.rates), t.angles, t.exposed, t.peripodial)
            x, rc, st = s.runOneStep(x, t.dt)
            assert rc == capi.TF_OK
            fg, _ = s.get_growth()
            _check(fg.reshape(-1, 9), z["frames"][step], step)
        np.testing.assert_array_equal(x, t.x)  # every DoF fixed: the mechanics never moved a node
