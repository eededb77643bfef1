"""Meshes of MeshBlocks on one GPU: ghost zones between blocks filled by the
device exchange between RK stages (Athena's SEND_HYD / RECV_HYD / SETB_HYD).

Every cell's arithmetic is the same whichever block holds it, and the ghost
exchange copies the neighbours' values exactly, so an FP64 mesh reproduces
the single block of the same domain bit for bit (the mesh-wide CFL minimum
is the single block's minimum); against the oracle the step carries the FP64
bar of the per-step parity tests.  The FP32 path's reference pressure is the
mesh-wide level mean, summed in a different order than the single block's,
so a mixed-precision mesh agrees with the single block to the FP32 path's
own error (1e-9 of the state after a few steps).
"""
import ctypes

import numpy as np
import pytest

from canoe_b200 import Mesh, MeshBlock, problems
from canoe_b200._abi import BC_BLOCK, CanoeError, FP32_PERTURBATION, check, load
from conftest import max_var_rel_l2, rel_l2
from test_gpu_parity import perturb

pytestmark = pytest.mark.gpu


def _c2(**kw):
    args = dict(nx1=24, nx2=16, nx3=12, x1max=3000.0, x2max=4000.0, x3max=3000.0, noise=0.5)
    args.update(kw)
    return problems.moist3d(**args)


def _c1():
    return problems.bubble2d(nx1=40, nx2=24, x1max=400.0, x2max=240.0)


CASES = {
    "c2_periodic_2x2": (lambda: perturb(_c2(), dv=0.5), 2, 2),
    "c2_periodic_4x3": (lambda: perturb(_c2(), dv=0.5), 4, 3),
    "c2_full5x5_2x1": (lambda: perturb(_c2(implicit_flag=9), dv=0.5), 2, 1),
    "c1_walls_3x1": (lambda: perturb(_c1(), dv=0.5), 3, 1),
}


@pytest.mark.parametrize("graph", [False, True], ids=["launches", "graph"])
@pytest.mark.parametrize("case", list(CASES))
def test_mesh_reproduces_single_block(case, graph):
    make, nb2, nb3 = CASES[case]
    p = make()
    one = MeshBlock(p)
    m = Mesh(p, nb2, nb3, graph=graph)
    assert m.new_dt() == one.new_dt()
    for _ in range(3):
        one.step()
        m.step()
    ref = p.interior(one.conserved())
    got = p.interior(m.conserved())
    assert one.error_word() == 0 and m.error_word() == 0
    assert np.array_equal(got, ref), float(np.abs(got - ref).max())
    assert m.new_dt() == one.new_dt()
    m.close()
    one.close()


def test_mesh_matches_oracle(oracle_mod):
    p = perturb(_c2(), dv=0.5)
    ora = oracle_mod.OracleBlock(p)
    m = Mesh(p, 2, 2)
    for _ in range(2):
        dt = ora.new_dt()
        assert abs(m.new_dt() - dt) <= 1e-12 * dt
        ora.step(dt)
        m.step(dt)
    a, b = p.interior(m.conserved()), p.interior(ora.conserved())
    assert rel_l2(a, b) < 1e-11
    ny = p.ny
    wn = np.linalg.norm(b[1:1 + ny].sum(axis=0))
    per = [rel_l2(a[n], b[n], floor=(wn if 1 <= n <= ny else 1e-12 * np.linalg.norm(b)))
           for n in range(b.shape[0])]
    assert max(per) < 5e-11, per
    m.close()


def test_per_stage_api_matches_mesh_step():
    """canoe_block_stage + canoe_block_exchange_ghosts driven by the host (the
    reference's per-stage task list) gives the mesh step's bits; the host
    takes the mesh-wide dt as the minimum of the blocks' own CFL steps."""
    lib = load()
    p = perturb(_c2(), dv=0.5)
    m = Mesh(p, 2, 2)
    h = Mesh(p, 2, 2)  # its blocks are driven stage by stage below
    for _ in range(2):
        dt = min(b.new_dt() for b in h.blocks)
        assert dt == m.new_dt()
        for s in range(3):
            for b in h.blocks:
                check(lib.canoe_block_stage(b.h, s, dt if s == 0 else -1.0), "stage")
            for b in h.blocks:
                b.synchronize()
            for b in h.blocks:
                check(lib.canoe_block_exchange_ghosts(b.h), "exchange")
            for b in h.blocks:
                b.synchronize()
        m.step()
    assert np.array_equal(h.conserved(), m.conserved())
    m.close()
    h.close()


def test_mixed_precision_mesh_near_single_block():
    p = perturb(_c2(), dv=0.5)
    p.cfg.precision = FP32_PERTURBATION
    one = MeshBlock(p)
    m = Mesh(p, 2, 2)
    dt = one.new_dt()
    for _ in range(3):
        one.step(dt)
        m.step(dt)
    a, b = p.interior(m.conserved()), p.interior(one.conserved())
    assert rel_l2(a, b) < 1e-9
    m.close()
    one.close()


def test_block_sides_need_the_mesh():
    lib = load()
    p = _c2()
    p.cfg.bc[3] = BC_BLOCK
    b = MeshBlock(p)
    # a lone step would leave the block side's ghosts unfilled
    with pytest.raises(CanoeError):
        b.step()
    # exchange without a neighbour is refused
    assert lib.canoe_block_exchange_ghosts(b.h) != 0
    # a neighbour must share nx1
    q = _c2(nx1=20, x1max=2500.0)
    other = MeshBlock(q)
    assert lib.canoe_block_set_neighbor(b.h, 3, other.h) != 0
    # x1 cannot be a block side
    r = _c2()
    r.cfg.bc[1] = BC_BLOCK
    with pytest.raises(CanoeError):
        MeshBlock(r)
    b.close()
    other.close()


def test_distributed_driver_on_one_gpu_reproduces_single_block():
    """canoe_b200.distributed with every block on this GPU: the ghost slabs
    travel through canoe_block_pack_side / canoe_block_unpack_side (the
    buffers a multi-GPU run hands to NCCL) and the step equals the single
    block's bit for bit."""
    from canoe_b200 import distributed
    p = perturb(_c2(), dv=0.5)
    one = MeshBlock(p)
    dm = distributed.DistributedMesh.from_domain(p, 2, 2)
    assert dm.dt == one.new_dt()
    for _ in range(3):
        dt = dm.step()
        one.step(dt)
    from canoe_b200 import partition
    got = partition.gather(dm_split(p, 2, 2), p.u.shape,
                           [dm.conserved(q) for q in range(4)], p.cfg.nx2, p.cfg.nx3)
    assert np.array_equal(p.interior(got), p.interior(one.conserved()))
    assert dm.dt == one.new_dt()
    dm.close()
    one.close()


def dm_split(p, nb2, nb3):
    from canoe_b200 import partition
    return partition.split(p, nb2, nb3)
