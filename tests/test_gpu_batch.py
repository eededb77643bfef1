"""Batched uneven blocks: a batch step is each block's own step, whether the
batch runs as one CUDA graph or as plain launches, and the autotuned
threads per x1 pencil change no result (every loop strides by the block
size, each row's arithmetic is the same)."""
import numpy as np
import pytest

from canoe_b200 import Batch, MeshBlock, problems

pytestmark = pytest.mark.gpu


def _problems():
    return problems.batch_c5(nblocks=3, nz=(16, 40), nh=(6, 12), seed=11)


def _reference(ps, dt, nsteps):
    out = []
    for p in ps:
        b = MeshBlock(p)
        b.set_fixed_dt(dt)
        for _ in range(nsteps):
            b.step()
        out.append(b.conserved())
        b.close()
    return out


@pytest.mark.parametrize("graph", [True, False])
def test_batch_equals_blocks(graph):
    ps = _problems()
    dt = 0.5
    ref = _reference(ps, dt, 2)
    blocks = [MeshBlock(p) for p in ps]
    for b in blocks:
        b.set_fixed_dt(dt)
    bt = Batch(blocks, graph=graph)
    bt.step()
    bt.step()
    bt.synchronize()
    for b, r in zip(blocks, ref):
        assert np.array_equal(b.conserved(), r)


def test_autotune_keeps_state_and_results():
    ps = _problems()
    dt = 0.5
    ref = _reference(ps, dt, 2)
    blocks = [MeshBlock(p) for p in ps]
    for b in blocks:
        b.set_fixed_dt(dt)
    u0 = [b.conserved() for b in blocks]
    bt = Batch(blocks)
    choice = bt.autotune()
    assert all(c in (64, 96, 128, 160) for c in choice)
    for b, u in zip(blocks, u0):
        assert np.array_equal(b.conserved(), u)
    bt.step()
    bt.step()
    bt.synchronize()
    for b, r in zip(blocks, ref):
        assert np.array_equal(b.conserved(), r)
