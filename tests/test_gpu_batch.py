"""GPU tests of the batched mode: many independent tissues of uneven size in one context.

Each tissue must follow exactly the single-tissue path (its own Newton convergence and cap):
positions after the steps within 1e-9 of the tissue size of separate single-tissue runs and of
the oracle, and the same Newton iteration counts.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tissueorigami_b200 import capi, mesh
from tissueorigami_b200.newton import BatchSolver, NewtonRaphsonSolver

pytestmark = pytest.mark.gpu


def _tissues():
    out = []
    for k, n in enumerate([400, 1500, 700, 3000, 500, 2200]):
        E = 600.0 + 400.0 * k
        out.append(mesh.small_disc(100 + k, n, E, n_steps=3) if k % 2 == 0 else mesh.small_rect_sized(100 + k, n, E, n_steps=3))
    return out


@pytest.mark.parametrize("precond", ["two_level", "block_jacobi"])
def test_batch_matches_single_tissue_runs(precond):
    pc = {"two_level": capi.TF_PRECOND_TWO_LEVEL, "block_jacobi": capi.TF_PRECOND_BLOCK_JACOBI}[precond]
    ts = _tissues()
    n_steps = 3
    singles, its_single = [], []
    for t in ts:
        with NewtonRaphsonSolver.from_tissue(t, krylov_rtol=1e-14) as s:
            x = t.x.copy()
            its = []
            for _ in range(n_steps):
                x, rc, st = s.runOneStep(x, t.dt)
                assert rc == capi.TF_OK
                its.append(st["newton_iters"])
            singles.append(x)
            its_single.append(its)
    with BatchSolver(ts, krylov_rtol=1e-14, precond=pc) as b:
        assert b.preconditioner()[0] == pc
        assert b.smoother_block() == 2  # every tissue has two node surfaces: two-node columns
        x = b.join([t.x for t in ts])
        its_batch = [[] for _ in ts]
        for _ in range(n_steps):
            x, rc, st = b.runOneStep(x, ts[0].dt)
            assert rc == capi.TF_OK
            stats = b.tissue_stats()
            assert (stats["status"] == 0).all()
            for i in range(len(ts)):
                its_batch[i].append(int(stats["newton_iters"][i]))
        xs = b.split(x)
        pc_used, n_coarse, refreshes = b.preconditioner()
        if pc == capi.TF_PRECOND_TWO_LEVEL:
            # one coarse space per tissue: at least one aggregate (six modes) each
            assert n_coarse >= 6 * len(ts) and refreshes >= 1
        else:
            assert n_coarse == 0
    assert its_batch == its_single
    for t, xb, xsng in zip(ts, xs, singles):
        assert np.abs(xb - xsng).max() <= 1e-9 * t.size


@pytest.mark.parametrize("precond", ["two_level", "block_jacobi"])
def test_batch_tissue_matches_oracle(precond):
    pc = {"two_level": capi.TF_PRECOND_TWO_LEVEL, "block_jacobi": capi.TF_PRECOND_BLOCK_JACOBI}[precond]
    ts = _tissues()[:3]
    with BatchSolver(ts, krylov_rtol=1e-14, precond=pc) as b:
        x = b.join([t.x for t in ts])
        for _ in range(2):
            x, rc, st = b.runOneStep(x, ts[0].dt)
            assert rc == capi.TF_OK
        xs = b.split(x)
    x_ref, _, _, _ = O.simulate_sparse(ts[1], n_steps=2)
    assert np.abs(xs[1] - x_ref).max() <= 1e-9 * ts[1].size


def test_batch_assembly_is_block_diagonal():
    ts = _tissues()[:2]
    with BatchSolver(ts) as b:
        rowptr, colidx = b.pattern()
        tissue_of = np.repeat(np.arange(len(ts)), [t.n_nodes for t in ts])
        rows = np.repeat(np.arange(b.n_nodes), np.diff(rowptr))
        assert (tissue_of[rows] == tissue_of[colidx]).all()


def test_sharded_batch_matches_one_batch():
    """Two ranks' shards (run here one after the other on the one GPU, as two independent
    contexts: nothing waits on anything) give the positions of the whole batch in one context,
    within 1e-9 of each tissue's size."""
    from tissueorigami_b200.sharding import ShardedBatch

    ts = _tissues()
    with BatchSolver(ts, krylov_rtol=1e-14) as b:
        x = b.join([t.x for t in ts])
        for _ in range(2):
            x, rc, _ = b.runOneStep(x, ts[0].dt)
            assert rc == capi.TF_OK
        whole = b.split(x)
    merged = {}
    for rank in range(2):
        sb = ShardedBatch(ts, rank, 2, lambda tl: BatchSolver(tl, krylov_rtol=1e-14))
        try:
            local, stats = sb.run(2, ts[0].dt)
            assert all(s["rc"] == capi.TF_OK for s in stats)
            assert not (set(local) & set(merged))
            merged.update(local)
        finally:
            sb.close()
    assert sorted(merged) == list(range(len(ts)))
    for i, t in enumerate(ts):
        assert np.abs(merged[i] - whole[i]).max() <= 1e-9 * t.size


def test_batch_node_blocks_match_column_blocks():
    """The batch with 3x3 node blocks and with two-node column blocks: the same positions within
    1e-9 of each tissue's size and the same Newton iteration counts."""
    ts = _tissues()[:4]
    out = {}
    for sn in (1, 0):
        with BatchSolver(ts, krylov_rtol=1e-14, smoother_nodes=sn) as b:
            assert b.smoother_block() == (1 if sn == 1 else 2)
            x = b.join([t.x for t in ts])
            its = []
            for _ in range(2):
                x, rc, _ = b.runOneStep(x, ts[0].dt)
                assert rc == capi.TF_OK
                its.append(b.tissue_stats()["newton_iters"].tolist())
            out[sn] = (b.split(x), its)
    assert out[0][1] == out[1][1]
    for t, a, c in zip(ts, out[1][0], out[0][0]):
        assert np.abs(a - c).max() <= 1e-9 * t.size
