"""A domain stepped as a mesh of MeshBlocks resident on one GPU (C ABI
canoe_block_set_neighbor / canoe_mesh_*): Athena's Mesh driving the task
list of every block per RK stage with the boundary exchange between stages
(main.cpp:119-121, patches/24.time_integrator.patch:17-19).

    m = Mesh(problem, nb2=2, nb3=2)   # the domain cut into 2 x 2 blocks
    m.step()                          # mesh-wide CFL dt, ghosts exchanged
    u = m.conserved()                 # gathered into the domain's layout
"""
import ctypes

import numpy as np

from . import partition
from ._abi import check, load
from .block import MeshBlock


class Mesh:
    def __init__(self, problem, nb2, nb3=1, graph=False):
        self.lib = load()
        self.problem = problem
        self.split = partition.split(problem, nb2, nb3)
        self.blocks = [MeshBlock(p) for p in self.split.blocks]
        for b, nbr in zip(self.blocks, self.split.neighbors):
            for side, q in nbr.items():
                check(self.lib.canoe_block_set_neighbor(b.h, side, self.blocks[q].h),
                      "canoe_block_set_neighbor")
        arr = (ctypes.c_void_p * len(self.blocks))(*[b.h.value for b in self.blocks])
        h = ctypes.c_void_p()
        check(self.lib.canoe_mesh_create(arr, len(self.blocks), ctypes.byref(h)),
              "canoe_mesh_create")
        self.h = h
        if graph:
            check(self.lib.canoe_mesh_use_graph(h, 1), "canoe_mesh_use_graph")

    def close(self):
        if self.h:
            self.lib.canoe_mesh_destroy(self.h)
            self.h = None
        for b in self.blocks:
            b.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt=-1.0):
        check(self.lib.canoe_mesh_step(self.h, float(dt)), "canoe_mesh_step")

    def new_dt(self):
        d = ctypes.c_double()
        check(self.lib.canoe_mesh_new_dt(self.h, ctypes.byref(d)), "canoe_mesh_new_dt")
        return d.value

    def synchronize(self):
        check(self.lib.canoe_mesh_synchronize(self.h), "synchronize")

    def error_word(self):
        bits = 0
        for b in self.blocks:
            bits |= b.error_word()
        return bits

    def conserved(self):
        self.synchronize()
        c = self.problem.cfg
        return partition.gather(self.split, self.problem.u.shape,
                                [b.conserved() for b in self.blocks], c.nx2, c.nx3)
