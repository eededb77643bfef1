"""Batches of uneven MeshBlocks stepped together (C ABI canoe_batch_*).

    bt = Batch([MeshBlock(p) for p in problems.batch_c5()])
    bt.autotune()       # threads per x1 pencil, per block
    bt.step()           # one step of every block: one CUDA graph launch

Each block keeps its own state and dt (set_fixed_dt or its CFL step).
"""
import ctypes

import numpy as np

from ._abi import check, load


class Batch:
    def __init__(self, blocks, graph=True):
        self.lib = load()
        self.blocks = list(blocks)
        arr = (ctypes.c_void_p * len(self.blocks))(*[b.h.value for b in self.blocks])
        h = ctypes.c_void_p()
        check(self.lib.canoe_batch_create(arr, len(self.blocks), ctypes.byref(h)),
              "canoe_batch_create")
        self.h = h
        self.use_graph(graph)

    def close(self):
        if self.h:
            self.lib.canoe_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def use_graph(self, on=True):
        check(self.lib.canoe_batch_use_graph(self.h, 1 if on else 0), "use_graph")

    def step(self):
        check(self.lib.canoe_batch_step(self.h), "canoe_batch_step")

    def synchronize(self):
        check(self.lib.canoe_batch_synchronize(self.h), "synchronize")

    def autotune(self):
        out = np.zeros(len(self.blocks), dtype=np.int32)
        check(self.lib.canoe_batch_autotune(self.h, out.ctypes.data), "canoe_batch_autotune")
        return out

    def shapes(self):
        """(threads per x1 pencil, cells per x2 / x3 flux run) of every block
        (0 = the default)."""
        import ctypes
        out = []
        for b in self.blocks:
            t, r = ctypes.c_int32(0), ctypes.c_int32(0)
            check(self.lib.canoe_block_get_shapes(b.h, ctypes.byref(t), ctypes.byref(r)),
                  "canoe_block_get_shapes")
            out.append((t.value, r.value))
        return out
