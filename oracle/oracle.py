"""ctypes wrapper of the CPU oracle (oracle/lib/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference leg, as the checker.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_void_p

import numpy as np

from canoe_b200._abi import BlockConfig, SatOpts, ShellConfig, Thermo

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "lib", "liboracle.so")

_lib = None


def build():
    subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    sig = [
        ("oracle_last_error", c_char_p, []),
        ("oracle_set_threads", c_int, [c_int]),
        ("oracle_block_new", c_void_p, [POINTER(BlockConfig)]),
        ("oracle_block_free", None, [c_void_p]),
        ("oracle_block_set_roundtrip", None, [c_void_p, c_int]),
        ("oracle_block_set_diffusion", None, [c_void_p, c_double, c_double]),
        ("oracle_block_set_conserved", c_int, [c_void_p, c_void_p]),
        ("oracle_block_set_primitive", c_int, [c_void_p, c_void_p]),
        ("oracle_block_get_conserved", c_int, [c_void_p, c_void_p]),
        ("oracle_block_get_primitive", c_int, [c_void_p, c_void_p]),
        ("oracle_block_calculate_fluxes", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        ("oracle_block_solve_implicit", c_int, [c_void_p, c_void_p, c_double]),
        ("oracle_block_step", c_int, [c_void_p, c_double, c_int]),
        ("oracle_periodic_block_solve", c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p,
                                                c_void_p, c_void_p]),
        ("oracle_block_new_dt", c_double, [c_void_p]),
        ("oracle_block_stage", c_int, [c_void_p, c_int, c_double]),
        ("oracle_x1_change_to_temperature", c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p,
                                                    c_void_p, c_void_p]),
        ("oracle_x1_restore_from_temperature", c_int, [c_void_p, c_int, c_int, c_void_p,
                                                       c_void_p, c_void_p, c_int, c_int]),
        ("oracle_riemann", c_int, [c_int, POINTER(Thermo), c_int, c_void_p, c_void_p, c_void_p, c_int64]),
        ("oracle_cons_to_prim", c_int, [POINTER(Thermo), c_void_p, c_void_p, c_int64]),
        ("oracle_prim_to_cons", c_int, [POINTER(Thermo), c_void_p, c_void_p, c_int64]),
        ("oracle_satadj", c_int, [POINTER(Thermo), POINTER(SatOpts), c_void_p, c_int64, c_void_p,
                                  c_void_p, c_void_p, c_void_p]),
        ("oracle_mlp_forward", c_int, [c_void_p, c_int, c_void_p, c_int64, c_void_p]),
        ("oracle_mlp_loss_grad", c_double, [c_void_p, c_int, c_void_p, c_void_p, c_int64, c_void_p]),
        ("oracle_shell_new", c_void_p, [POINTER(ShellConfig)]),
        ("oracle_shell_free", None, [c_void_p]),
        ("oracle_shell_set_conserved", c_int, [c_void_p, c_void_p]),
        ("oracle_shell_set_primitive", c_int, [c_void_p, c_void_p]),
        ("oracle_shell_get", c_int, [c_void_p, c_int, c_void_p]),
        ("oracle_shell_fill_ghosts", c_int, [c_void_p]),
        ("oracle_shell_cons_to_prim", c_int, [c_void_p]),
        ("oracle_shell_prim_to_cons", c_int, [c_void_p]),
        ("oracle_shell_calculate_fluxes", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        ("oracle_shell_step", c_int, [c_void_p, c_double, c_int]),
    ]
    for name, res, args in sig:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data if a is not None else None


def set_threads(n):
    return load().oracle_set_threads(n)


class OracleBlock:
    """The oracle's MeshBlock (FP64, OpenMP)."""

    def __init__(self, problem, roundtrip=True):
        self.lib = load()
        self.problem = problem
        self.h = self.lib.oracle_block_new(ctypes.byref(problem.cfg))
        if not self.h:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        self.lib.oracle_block_set_roundtrip(self.h, 1 if roundtrip else 0)
        self.shape = problem.u.shape
        self.set_conserved(problem.u)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_block_free(self.h)
            self.h = None

    def set_conserved(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.shape == self.shape
        self.lib.oracle_block_set_conserved(self.h, u.ctypes.data)

    def set_diffusion(self, K, p0=1.0e5):
        self.lib.oracle_block_set_diffusion(self.h, float(K), float(p0))

    def set_primitive(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        self.lib.oracle_block_set_primitive(self.h, w.ctypes.data)

    def conserved(self):
        out = np.empty(self.shape)
        self.lib.oracle_block_get_conserved(self.h, out.ctypes.data)
        return out

    def primitive(self):
        out = np.empty(self.shape)
        self.lib.oracle_block_get_primitive(self.h, out.ctypes.data)
        return out

    def calculate_fluxes(self):
        nv, n3, n2, n1 = self.shape
        f1 = np.zeros((nv, n3, n2, n1 + 1))
        f2 = np.zeros((nv, n3, n2 + 1, n1))
        f3 = np.zeros((nv, n3 + 1, n2, n1))
        rc = self.lib.oracle_block_calculate_fluxes(self.h, f1.ctypes.data, f2.ctypes.data,
                                                    f3.ctypes.data)
        assert rc == 0, self.lib.oracle_last_error().decode()
        return f1, f2, f3

    def solve_implicit(self, du, dt):
        d = np.ascontiguousarray(du, dtype=np.float64).copy()
        rc = self.lib.oracle_block_solve_implicit(self.h, d.ctypes.data, float(dt))
        assert rc == 0, self.lib.oracle_last_error().decode()
        return d

    def step(self, dt=-1.0, nsteps=1):
        rc = self.lib.oracle_block_step(self.h, float(dt), int(nsteps))
        assert rc == 0, self.lib.oracle_last_error().decode()

    def new_dt(self):
        return self.lib.oracle_block_new_dt(self.h)

    def stage(self, stage, dt):
        """one RK stage of the oracle's step (ghosts of block sides untouched)"""
        rc = self.lib.oracle_block_stage(self.h, stage, float(dt))
        assert rc == 0, self.lib.oracle_last_error().decode()

    def x1_change_to_temperature(self, k, j):
        """The x1 hydrostatic decomposition of column (k, j) of the current
        primitive state: (q (nv, nc1) decomposed, psf, psv, gamma)."""
        nv, nc1 = self.shape[0], self.shape[3]
        q = np.zeros((nv, nc1))
        psf = np.zeros(nc1 + 1)
        psv = np.zeros(nc1)
        gam = np.zeros(nc1)
        self.lib.oracle_x1_change_to_temperature(self.h, k, j, q.ctypes.data, psf.ctypes.data,
                                                 psv.ctypes.data, gam.ctypes.data)
        return q, psf, psv, gam

    def x1_restore_from_temperature(self, k, j, q, wl, wr, lo, hi):
        """Its inverse with the column's arrays of the last call above:
        returns (q, wl, wr) restored; wl / wr (nv, nc1 + 1), faces lo..hi."""
        q = np.array(q, dtype=np.float64, order="C")
        wl = np.array(wl, dtype=np.float64, order="C")
        wr = np.array(wr, dtype=np.float64, order="C")
        self.lib.oracle_x1_restore_from_temperature(self.h, k, j, q.ctypes.data, wl.ctypes.data,
                                                    wr.ctypes.data, lo, hi)
        return q, wl, wr


def periodic_block_solve(a, b, c, rhs):
    """The oracle's El-Mikkawy cyclic block-tridiagonal solve.  a, b, c:
    (n + 1, N, N) blocks of rows 0..n, of which rows 1..n are the system and
    c[0] the lower corner (row n's coupling to row 1); rhs (n + 1, N).
    Returns x (n + 1, N) with row 0 zero."""
    a, b, c, rhs = (np.ascontiguousarray(v, dtype=np.float64) for v in (a, b, c, rhs))
    n, nb = a.shape[0] - 1, a.shape[1]
    x = np.zeros_like(rhs)
    rc = load().oracle_periodic_block_solve(nb, n, _p(a), _p(b), _p(c), _p(rhs), _p(x))
    if rc:
        raise ValueError("periodic_block_solve: unsupported block size or n < 3")
    return x


def riemann(rsolver, th, ivx, wl, wr):
    wl = np.ascontiguousarray(wl, dtype=np.float64)
    wr = np.ascontiguousarray(wr, dtype=np.float64)
    flx = np.zeros_like(wl)
    load().oracle_riemann(rsolver, ctypes.byref(th), ivx, wl.ctypes.data, wr.ctypes.data,
                          flx.ctypes.data, wl.shape[1])
    return flx


def cons_to_prim(th, u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    w = np.zeros_like(u)
    load().oracle_cons_to_prim(ctypes.byref(th), u.ctypes.data, w.ctypes.data, u.shape[1])
    return w


def prim_to_cons(th, w):
    w = np.ascontiguousarray(w, dtype=np.float64)
    u = np.zeros_like(w)
    load().oracle_prim_to_cons(ctypes.byref(th), w.ctypes.data, u.ctypes.data, w.shape[1])
    return u


def satadj(th, u, tol=1e-8, max_iter=30, t_guess=None, mode=None):
    """Saturation adjustment of cells u (NV, n) in place; returns T, iters
    (evaluations of f), flags.  mode: 0 cold, 1 start at t_guess, 2 hybrid
    (default 1 when t_guess is given, else 0)."""
    assert u.flags.c_contiguous and u.dtype == np.float64
    n = u.shape[1]
    if mode is None:
        mode = 1 if t_guess is not None else 0
    o = SatOpts(tol, max_iter, mode)
    t = np.zeros(n)
    it = np.zeros(n, dtype=np.int32)
    fl = np.zeros(n, dtype=np.int32)
    tg = None if t_guess is None else np.ascontiguousarray(t_guess, dtype=np.float64)
    load().oracle_satadj(ctypes.byref(th), ctypes.byref(o), u.ctypes.data, n, _p(tg),
                         t.ctypes.data, it.ctypes.data, fl.ctypes.data)
    return t, it, fl


def mlp_forward(params, nh, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    y = np.zeros(x.shape[0])
    load().oracle_mlp_forward(p.ctypes.data, nh, x.ctypes.data, x.shape[0], y.ctypes.data)
    return y


def mlp_loss_grad(params, nh, x, y):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    g = np.zeros_like(p)
    loss = load().oracle_mlp_loss_grad(p.ctypes.data, nh, x.ctypes.data, y.ctypes.data,
                                       x.shape[0], g.ctypes.data)
    return loss, g


class OracleShell:
    """The oracle's six-panel cubed-sphere shell (FP64)."""

    def __init__(self, problem):
        self.lib = load()
        self.problem = problem
        self.h = self.lib.oracle_shell_new(ctypes.byref(problem.cfg))
        if not self.h:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        self.shape = problem.u.shape
        self.set_conserved(problem.u)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_shell_free(self.h)
            self.h = None

    def _check(self, rc):
        assert rc == 0, self.lib.oracle_last_error().decode()

    def set_conserved(self, u, fill=True):
        """load u; by default fill the panel ghosts and compute w"""
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.shape == self.shape
        self.lib.oracle_shell_set_conserved(self.h, u.ctypes.data)
        if fill:
            self.fill_ghosts()
            self.cons_to_prim()

    def fill_ghosts(self):
        self._check(self.lib.oracle_shell_fill_ghosts(self.h))

    def cons_to_prim(self):
        self._check(self.lib.oracle_shell_cons_to_prim(self.h))

    def conserved(self):
        out = np.empty(self.shape)
        self.lib.oracle_shell_get(self.h, 0, out.ctypes.data)
        return out

    def primitive(self):
        out = np.empty(self.shape)
        self.lib.oracle_shell_get(self.h, 1, out.ctypes.data)
        return out

    def calculate_fluxes(self):
        six, nv, n3, n2, n1 = self.shape
        f1 = np.zeros((6, nv, n3, n2, n1 + 1))
        f2 = np.zeros((6, nv, n3, n2 + 1, n1))
        f3 = np.zeros((6, nv, n3 + 1, n2, n1))
        self._check(self.lib.oracle_shell_calculate_fluxes(self.h, f1.ctypes.data,
                                                           f2.ctypes.data, f3.ctypes.data))
        return f1, f2, f3

    def step(self, dt, nsteps=1):
        self._check(self.lib.oracle_shell_step(self.h, float(dt), int(nsteps)))
