"""A domain split across GPUs: one process (rank) per GPU, the MeshBlocks of
each rank resident on its GPU, ghost slabs exchanged between RK stages.

This is Athena's Mesh over MPI ranks for this path: every rank runs the
per-stage task list of its blocks (src/tasklist/implicit_hydro_tasks.cpp),
the boundary tasks SEND_HYD / RECV_HYD / SETB_HYD move the NGHOST ghost
layers of every block side between stages (patches/24.time_integrator.patch:
17-19), and Mesh::NewTimeStep takes the minimum CFL step over all blocks.
The domain is cut in x2 / x3 only (canoe_b200.partition): x1, the vertical,
stays whole, so the hydrostatic scan and the implicit column solve need no
messages.

    dm = DistributedMesh.from_domain(problem, nb2, nb3, dist)  # torch.distributed up
    dm.step()              # every stage of the rank's blocks, ghosts exchanged
    u = dm.conserved(q)    # the state of a block this rank owns

Messages: for every block side with a neighbour, the neighbour packs its
interior layers next to the shared side (canoe_block_pack_side) and the
block unpacks them into its ghosts (canoe_block_unpack_side).  Both ranks
enumerate the messages in the same global order (receiver block, side), so
the point-to-point operations of one batch match pairwise in order, as NCCL
requires; a message between two blocks of one rank is a device copy.
The step dt is one all-reduce (MIN) of one double per step.

A backend holds the blocks: GpuBackend (the CUDA library, one GPU per rank,
NCCL) here; the tests drive the same exchange logic with the CPU oracle and
gloo.
"""
import ctypes

from . import partition

OPPOSITE = {2: 3, 3: 2, 4: 5, 5: 4}


class GpuBackend:
    """Blocks of the CUDA library on this rank's GPU, every launch on
    torch's current stream so that NCCL transfers order after the packs and
    before the unpacks."""

    def __init__(self):
        import torch
        self.torch = torch
        from ._abi import check, load
        self.lib = load()
        self.check = check
        self.stream = torch.cuda.current_stream()

    def make(self, problem):
        from .block import MeshBlock
        b = MeshBlock(problem)
        self.check(self.lib.canoe_block_set_stream(b.h, ctypes.c_void_p(self.stream.cuda_stream)),
                   "canoe_block_set_stream")
        return b

    def side_buffer(self, b, side):
        n = ctypes.c_int64()
        self.check(self.lib.canoe_block_side_doubles(b.h, side, ctypes.byref(n)), "side_doubles")
        return self.torch.empty(n.value, dtype=self.torch.float64, device="cuda")

    def pack(self, b, side, buf):
        self.check(self.lib.canoe_block_pack_side(b.h, side, buf.data_ptr()), "pack_side")

    def unpack(self, b, side, buf):
        self.check(self.lib.canoe_block_unpack_side(b.h, side, buf.data_ptr()), "unpack_side")

    def stage(self, b, stage, dt):
        self.check(self.lib.canoe_block_stage(b.h, stage, float(dt)), "canoe_block_stage")

    def new_dt(self, b):
        return b.new_dt()

    def dt_tensor(self, v):
        return self.torch.tensor([v], dtype=self.torch.float64, device="cuda")

    def conserved(self, b):
        return b.conserved()

    def close(self, b):
        b.close()


class DistributedMesh:
    def __init__(self, blocks, neighbors, owner, backend, dist=None):
        """blocks: {q: Problem} of every block (only the rank's own are
        built); neighbors: per block q {side: neighbour index}; owner: the
        rank of every block; dist: torch.distributed (None: one rank)."""
        self.dist = dist
        self.rank = dist.get_rank() if dist is not None else 0
        self.world = dist.get_world_size() if dist is not None else 1
        self.owner = list(owner)
        self.backend = backend
        self.local = [q for q in range(len(self.owner)) if self.owner[q] == self.rank]
        self.blocks = {q: backend.make(blocks[q]) for q in self.local}
        # every message of the mesh, in one global order: (receiver, side,
        # sender); the sender packs its side facing the receiver
        self.msgs = sorted((q, s, p) for q in range(len(self.owner))
                           for s, p in neighbors[q].items())
        self.bufs = {}
        for q, s, p in self.msgs:
            if self.owner[q] == self.rank:
                self.bufs[(q, s, "r")] = backend.side_buffer(self.blocks[q], s)
            if self.owner[p] == self.rank:
                self.bufs[(q, s, "s")] = backend.side_buffer(self.blocks[p], OPPOSITE[s])
        self.exchange()
        self.dt = self.mesh_dt()

    @classmethod
    def from_domain(cls, problem, nb2, nb3=1, dist=None, backend=None):
        """Cut a domain Problem into nb2 x nb3 blocks dealt to the ranks in
        contiguous ranges of block index."""
        sp = partition.split(problem, nb2, nb3)
        world = dist.get_world_size() if dist is not None else 1
        nb = len(sp.blocks)
        if nb < world:
            raise ValueError("fewer blocks than ranks")
        owner = [q * world // nb for q in range(nb)]
        return cls(dict(enumerate(sp.blocks)), sp.neighbors, owner, backend or GpuBackend(), dist)

    def exchange(self):
        """SEND_HYD / RECV_HYD / SETB_HYD of every block side of this rank."""
        ops, unpack = [], []
        for q, s, p in self.msgs:
            mine_q, mine_p = self.owner[q] == self.rank, self.owner[p] == self.rank
            if mine_p:
                sbuf = self.bufs[(q, s, "s")]
                self.backend.pack(self.blocks[p], OPPOSITE[s], sbuf)
            if mine_q and mine_p:
                self.backend.unpack(self.blocks[q], s, sbuf)
            elif mine_p:
                ops.append(self.dist.P2POp(self.dist.isend, sbuf, self.owner[q]))
            elif mine_q:
                rbuf = self.bufs[(q, s, "r")]
                ops.append(self.dist.P2POp(self.dist.irecv, rbuf, self.owner[p]))
                unpack.append((q, s, rbuf))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
        for q, s, rbuf in unpack:
            self.backend.unpack(self.blocks[q], s, rbuf)

    def mesh_dt(self):
        """Mesh::NewTimeStep: the minimum of every block's CFL step."""
        v = min(self.backend.new_dt(self.blocks[q]) for q in self.local)
        if self.dist is None:
            return v
        t = self.backend.dt_tensor(v)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        return float(t.item())

    def step(self, dt=None, update_dt=True):
        """One RK3 step of every block of this rank (dt: the mesh CFL step
        of the current state when None).  update_dt=False skips the mesh-wide
        CFL reduction after the step (a run with a fixed dt)."""
        dt = self.dt if dt is None else dt
        for s in range(3):
            for q in self.local:
                self.backend.stage(self.blocks[q], s, dt if s == 0 else -1.0)
            self.exchange()
        if update_dt:
            self.dt = self.mesh_dt()
        return dt

    def conserved(self, q):
        return self.backend.conserved(self.blocks[q])

    def close(self):
        for b in self.blocks.values():
            self.backend.close(b)
        self.blocks = {}
