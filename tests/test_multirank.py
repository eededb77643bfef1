"""The multi-rank paths on CPU: two gloo ranks on 127.0.0.1.

- bench.py's timing: every rank times its region with CUDA events and rank 0
  reports the whole-job rate from the slowest rank's time;
- the partitioned domain (canoe_b200.distributed): blocks dealt to ranks,
  ghost slabs exchanged between RK stages, the CFL step min-reduced."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms, rates = bench.job_rates([10.0 + rank, 20.0 - rank], 1000, 5, dist, device="cpu")
    out.put((rank, ms, rates))
    dist.barrier()
    dist.destroy_process_group()


def test_job_rates_take_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rates in res:
        assert ms == [11.0, 20.0]  # max over ranks of each region
        assert rates[0] == pytest.approx(world * 1000 * 5 / 11e-3)
        assert rates[1] == pytest.approx(world * 1000 * 5 / 20e-3)


def test_single_rank_without_process_group():
    import bench
    ms, rates = bench.job_rates([4.0], 10, 2, None, device="cpu")
    assert ms == [4.0] and rates == [pytest.approx(10 * 2 / 4e-3)]


# ---------------------------------------------------------------------------
# The partitioned data path (canoe_b200.distributed) with the oracle's blocks
# on CPU and gloo: two ranks, each owning blocks of a domain cut in x2 and
# x3, exchange ghost slabs between RK stages and min-reduce the CFL step.
# Every cell's arithmetic is the same whichever block holds it, so the
# partitioned run reproduces the single-block oracle run bit for bit.  The
# oracle's blocks run without writing the decomposition's round trip back
# into w (as the CUDA path computes): with it, a block's x2 / x3 fluxes would
# read its own interior after the x1 pass's round trip but its ghosts from
# before the neighbour's, an ulp-level dependence on where the cuts fall.

class OracleBackend:
    """The exchange logic of DistributedMesh over the oracle's blocks: slabs
    are numpy slices of the primitive state laid out as the CUDA library's
    pack buffers (variable, k, j, i)."""

    NG = 3

    def __init__(self):
        from oracle import oracle
        self.oracle = oracle
        self.dt = None

    def make(self, problem):
        return self.oracle.OracleBlock(problem, roundtrip=False)

    def _sl(self, b, side, ghosts):
        c = b.problem.cfg
        ng = self.NG
        ks, ke = (ng, ng + c.nx3 - 1) if c.nx3 > 1 else (0, 0)
        js, je = (ng, ng + c.nx2 - 1) if c.nx2 > 1 else (0, 0)
        lo = side % 2 == 0
        if side < 4:
            j0 = (js - ng if lo else je + 1) if ghosts else (js if lo else je - ng + 1)
            return (slice(None), slice(ks, ke + 1), slice(j0, j0 + ng), slice(None))
        k0 = (ks - ng if lo else ke + 1) if ghosts else (ks if lo else ke - ng + 1)
        return (slice(None), slice(k0, k0 + ng), slice(js, je + 1), slice(None))

    def side_buffer(self, b, side):
        import torch
        w = b.primitive()
        return torch.zeros(w[self._sl(b, side, False)].size, dtype=torch.float64)

    def pack(self, b, side, buf):
        import torch
        buf.copy_(torch.from_numpy(np.ascontiguousarray(b.primitive()[self._sl(b, side, False)]).ravel()))

    def unpack(self, b, side, buf):
        w = b.primitive()
        sl = self._sl(b, side, True)
        w[sl] = buf.numpy().reshape(w[sl].shape)
        b.set_primitive(w)

    def stage(self, b, stage, dt):
        if stage == 0:
            self.dt = dt
        b.stage(stage, self.dt)

    def new_dt(self, b):
        return b.new_dt()

    def dt_tensor(self, v):
        import torch
        return torch.tensor([v], dtype=torch.float64)

    def conserved(self, b):
        return b.conserved()

    def close(self, b):
        pass


def _domain(name):
    from canoe_b200 import problems
    from test_gpu_parity import perturb
    if name == "c2":
        return perturb(problems.moist3d(nx1=16, nx2=12, nx3=12, x1max=2000.0, x2max=3000.0,
                                        x3max=3000.0, noise=0.5), dv=0.5)
    return perturb(problems.bubble2d(nx1=20, nx2=24, x1max=200.0, x2max=240.0), dv=0.5)


def _partitioned_rank(rank, world, port, name, nb2, nb3, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    from canoe_b200 import distributed, partition
    from oracle import oracle
    oracle.set_threads(1)
    p = _domain(name)
    dm = distributed.DistributedMesh.from_domain(p, nb2, nb3, dist, OracleBackend())
    dts = [dm.step() for _ in range(3)]
    mine = {q: dm.conserved(q) for q in dm.local}
    got = [None] * world
    dist.all_gather_object(got, mine)
    if rank == 0:
        states = {}
        for d in got:
            states.update(d)
        sp = partition.split(p, nb2, nb3)
        dom = partition.gather(sp, p.u.shape, [states[q] for q in range(len(states))],
                               p.cfg.nx2, p.cfg.nx3)
        out.put((dts, p.interior(dom)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("name,nb2,nb3", [("c2", 2, 2), ("c2", 4, 1), ("c1", 2, 1)])
def test_partitioned_oracle_reproduces_single_block(name, nb2, nb3):
    from oracle import oracle
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partitioned_rank, args=(r, world, port, name, nb2, nb3, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    dts, got = q.get(timeout=240)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p = _domain(name)
    ob = oracle.OracleBlock(p, roundtrip=False)
    ref_dts = []
    for _ in range(3):
        dt = ob.new_dt()
        ref_dts.append(dt)
        ob.step(dt)
    assert dts == ref_dts
    ref = p.interior(ob.conserved())
    assert np.array_equal(got, ref), float(np.abs(got - ref).max())
