"""Host-side mirror of canoe's MeshBlock for this path, over the C ABI.

    blk = MeshBlock(problem)          # MeshBlock + MeshBlock::Impl
    blk.step()                        # one RK3 step (task list, all stages)
    u = blk.conserved()               # Hydro::u  (NV, nc3, nc2, nc1)
    w = blk.primitive()               # Hydro::w
    f1, f2, f3 = blk.calculate_fluxes()   # Hydro::CalculateFluxes
    blk.solve_implicit(du, dt)        # ImplicitSolver::SolveImplicit3D

All computation is in the CUDA library; errors raise CanoeError.
"""
import ctypes

import numpy as np

from ._abi import CanoeError, check, load


class MeshBlock:
    def __init__(self, problem, graph=False):
        self.lib = load()
        self.problem = problem
        self._x1f = problem.x1f  # keeps cfg.h_x1f alive
        h = ctypes.c_void_p()
        check(self.lib.canoe_block_create(ctypes.byref(problem.cfg), ctypes.byref(h)),
              "canoe_block_create")
        self.h = h
        nv, n1, n2, n3 = (ctypes.c_int32() for _ in range(4))
        check(self.lib.canoe_block_dims(h, *(ctypes.byref(x) for x in (nv, n1, n2, n3))))
        self.shape = (nv.value, n3.value, n2.value, n1.value)
        if graph:
            check(self.lib.canoe_block_use_graph(h, 1))
        self.set_conserved(problem.u)

    def close(self):
        if self.h:
            self.lib.canoe_block_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_conserved(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != self.shape:
            raise CanoeError(f"conserved state has shape {u.shape}, expected {self.shape}")
        check(self.lib.canoe_block_set_conserved(self.h, u.ctypes.data), "set_conserved")

    def conserved(self):
        out = np.empty(self.shape)
        check(self.lib.canoe_block_get_conserved(self.h, out.ctypes.data), "get_conserved")
        return out

    def primitive(self):
        out = np.empty(self.shape)
        check(self.lib.canoe_block_get_primitive(self.h, out.ctypes.data), "get_primitive")
        return out

    def step(self, dt=-1.0):
        check(self.lib.canoe_block_step(self.h, float(dt)), "step")

    def set_mlp(self, net):
        """learned warm start of the saturation adjustment (None: off)"""
        self._net = net  # the network must outlive its use
        check(self.lib.canoe_block_set_mlp(self.h, net.h if net is not None else None),
              "set_mlp")

    def satadj_stats(self):
        """{cells, evaluations, fallbacks, not converged} since the last call"""
        s = np.zeros(4, dtype=np.uint64)
        check(self.lib.canoe_block_satadj_stats(self.h, s.ctypes.data), "satadj_stats")
        return s

    def set_diffusion(self, K, p0=1.0e5):
        """the dense sinking bubble's dissipation source (straka.cpp:125-190)"""
        check(self.lib.canoe_block_set_diffusion(self.h, float(K), float(p0)), "set_diffusion")

    def set_fixed_dt(self, dt):
        check(self.lib.canoe_block_set_fixed_dt(self.h, float(dt)), "set_fixed_dt")

    def synchronize(self):
        check(self.lib.canoe_block_synchronize(self.h), "synchronize")

    def new_dt(self):
        d = ctypes.c_double()
        check(self.lib.canoe_block_new_dt(self.h, ctypes.byref(d)), "new_dt")
        return d.value

    def error_word(self):
        b = ctypes.c_uint32()
        check(self.lib.canoe_block_error_word(self.h, ctypes.byref(b)), "error_word")
        return b.value

    def device_ptrs(self):
        du, dw = ctypes.c_void_p(), ctypes.c_void_p()
        check(self.lib.canoe_block_device_ptrs(self.h, ctypes.byref(du), ctypes.byref(dw)))
        return du.value, dw.value

    def calculate_fluxes(self):
        """Hydro::CalculateFluxes: returns the three face-flux arrays (host)."""
        import torch
        nv, n3, n2, n1 = self.shape
        f1 = torch.zeros((nv, n3, n2, n1 + 1), dtype=torch.float64, device="cuda")
        f2 = torch.zeros((nv, n3, n2 + 1, n1), dtype=torch.float64, device="cuda")
        f3 = torch.zeros((nv, n3 + 1, n2, n1), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        check(self.lib.canoe_block_calculate_fluxes(self.h, f1.data_ptr(), f2.data_ptr(),
                                                    f3.data_ptr()), "calculate_fluxes")
        return f1.cpu().numpy(), f2.cpu().numpy(), f3.cpu().numpy()

    def solve_implicit(self, du, dt):
        """ImplicitSolver::SolveImplicit3D on a host du (returns the corrected du)."""
        import torch
        d = torch.from_numpy(np.ascontiguousarray(du, dtype=np.float64)).cuda()
        torch.cuda.synchronize()
        check(self.lib.canoe_block_solve_implicit(self.h, d.data_ptr(), float(dt)),
              "solve_implicit")
        return d.cpu().numpy()
