"""Host-side mirror of canoe's cubed-sphere shell (CubedSphere + the six
panel MeshBlocks) over the C ABI.

    sh = Shell(problem)                 # problems.shell_c3(...)
    sh.step(dt)                         # one RK3 step of all panels
    u = sh.conserved()                  # (6, NV, nc3, nc2, nc1)
    sh.fill_ghosts()                    # panel ghost exchange (cs::PackData)
    f1, f2, f3 = sh.calculate_fluxes()  # Hydro::CalculateFluxes of each panel
"""
import ctypes

import numpy as np

from ._abi import CanoeError, check, load


class Shell:
    def __init__(self, problem, fill=True):
        self.lib = load()
        self.problem = problem
        self._x1f = problem.x1f
        h = ctypes.c_void_p()
        check(self.lib.canoe_shell_create(ctypes.byref(problem.cfg), ctypes.byref(h)),
              "canoe_shell_create")
        self.h = h
        nv, n1, n2, n3 = (ctypes.c_int32() for _ in range(4))
        check(self.lib.canoe_shell_dims(h, *(ctypes.byref(x) for x in (nv, n1, n2, n3))))
        self.shape = (6, nv.value, n3.value, n2.value, n1.value)
        self.set_conserved(problem.u, fill=fill)

    def close(self):
        if self.h:
            self.lib.canoe_shell_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_conserved(self, u, fill=True):
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != self.shape:
            raise CanoeError(f"shell state has shape {u.shape}, expected {self.shape}")
        check(self.lib.canoe_shell_set_conserved(self.h, u.ctypes.data, 1 if fill else 0),
              "canoe_shell_set_conserved")

    def conserved(self):
        out = np.empty(self.shape)
        check(self.lib.canoe_shell_get_conserved(self.h, out.ctypes.data), "get_conserved")
        return out

    def primitive(self):
        out = np.empty(self.shape)
        check(self.lib.canoe_shell_get_primitive(self.h, out.ctypes.data), "get_primitive")
        return out

    def fill_ghosts(self):
        check(self.lib.canoe_shell_fill_ghosts(self.h), "fill_ghosts")
        check(self.lib.canoe_shell_synchronize(self.h), "synchronize")

    def calculate_fluxes(self):
        import torch
        six, nv, n3, n2, n1 = self.shape
        f1 = torch.zeros((6, nv, n3, n2, n1 + 1), dtype=torch.float64, device="cuda")
        f2 = torch.zeros((6, nv, n3, n2 + 1, n1), dtype=torch.float64, device="cuda")
        f3 = torch.zeros((6, nv, n3 + 1, n2, n1), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        check(self.lib.canoe_shell_calculate_fluxes(self.h, f1.data_ptr(), f2.data_ptr(),
                                                    f3.data_ptr()), "calculate_fluxes")
        return f1.cpu().numpy(), f2.cpu().numpy(), f3.cpu().numpy()

    def step(self, dt):
        check(self.lib.canoe_shell_step(self.h, float(dt)), "canoe_shell_step")

    def synchronize(self):
        check(self.lib.canoe_shell_synchronize(self.h), "synchronize")

    def error_word(self):
        b = ctypes.c_uint32()
        check(self.lib.canoe_shell_error_word(self.h, ctypes.byref(b)), "error_word")
        return b.value
