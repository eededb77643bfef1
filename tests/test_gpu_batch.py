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
    assert all(c in (64, 96, 128, 160, 192, 256) for c in choice)
    assert all(t == c and r in (0, 8, 16, 32, 64) for (t, r), c in zip(bt.shapes(), choice))
    for b, u in zip(blocks, u0):
        assert np.array_equal(b.conserved(), u)
    bt.step()
    bt.step()
    bt.synchronize()
    for b, r in zip(blocks, ref):
        assert np.array_equal(b.conserved(), r)


@pytest.mark.parametrize("flag", [1, 9])
def test_column_threads_do_not_change_results(flag):
    """Any thread count per x1 pencil gives the same bits (3x3: 64..256; the
    5x5 solve always runs 224 threads)."""
    import ctypes
    from canoe_b200 import problems
    from canoe_b200._abi import check, load
    lib = load()
    out = []
    for nt in (0, 64, 160, 256):
        p = problems.moist3d(nx1=40, nx2=12, nx3=8, x1max=5000.0, x2max=3000.0,
                             x3max=2000.0, noise=0.5, implicit_flag=flag)
        b = MeshBlock(p)
        check(lib.canoe_block_set_column_threads(b.h, nt))
        b.step(1.0)
        b.step(1.0)
        out.append(b.conserved())
        assert b.error_word() == 0
        b.close()
    for o in out[1:]:
        assert np.array_equal(o, out[0])


@pytest.mark.parametrize("precision", [0, 1])
def test_flux_run_length_does_not_change_results(precision):
    """Any number of cells per x2 / x3 flux run gives the same bits, in FP64
    and on the FP32 flux path."""
    from canoe_b200 import problems
    from canoe_b200._abi import check, load
    lib = load()
    out = []
    for cells in (0, 4, 8, 16, 64):
        p = problems.moist3d(nx1=24, nx2=40, nx3=36, x1max=3000.0, x2max=4000.0,
                             x3max=3600.0, noise=0.5)
        p.cfg.precision = precision
        b = MeshBlock(p)
        check(lib.canoe_block_set_flux_run(b.h, cells))
        b.step(1.0)
        b.step(1.0)
        out.append(b.conserved())
        assert b.error_word() == 0
        b.close()
    for o in out[1:]:
        assert np.array_equal(o, out[0])


def test_flux_run_rejects_out_of_range():
    from canoe_b200 import problems
    from canoe_b200._abi import load
    lib = load()
    b = MeshBlock(problems.moist3d(nx1=16, nx2=8, nx3=8, x1max=2000.0, x2max=800.0,
                                   x3max=800.0))
    assert lib.canoe_block_set_flux_run(b.h, 3) != 0
    assert lib.canoe_block_set_flux_run(b.h, 257) != 0
    assert lib.canoe_block_set_flux_run(b.h, 0) == 0
    b.close()
