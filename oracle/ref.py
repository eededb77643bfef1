"""ctypes wrapper of the reference's own source files compiled into
oracle/_ref/ (see oracle/Makefile, target ref, and oracle/ref_harness.cpp).

TEST INFRASTRUCTURE ONLY: the checker that pins the oracle's restatement to
the reference's arithmetic.  It needs the reference source tree to build
(REF, default the mounted reference checkout); where that tree is absent and
the libraries were not built, available() is False.
"""
import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int64, c_void_p

import numpy as np

from canoe_b200._abi import Thermo

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REF = os.environ.get("CANOE_REFERENCE", "/root/reference")
UNITS = ("lmars", "hllc", "decomp", "implicit")
NHS = (5, 8)

_libs = {}


def _path(unit, nh):
    return os.path.join(OUT, f"libref_{unit}_nv{nh}.so")


def build():
    """Compile the reference units when the reference tree is present."""
    if not os.path.isdir(os.path.join(REF, "src")):
        return False
    subprocess.run(["make", "-C", HERE, "-s", "ref", f"REF={REF}"], check=True)
    return True


def available():
    if all(os.path.exists(_path(u, n)) for u in UNITS for n in NHS):
        return True
    try:
        return build()
    except subprocess.CalledProcessError:
        return False


def lib(unit, nh):
    key = (unit, nh)
    if key in _libs:
        return _libs[key]
    L = ctypes.CDLL(_path(unit, nh))
    L.ref_last_error.restype = c_char_p
    L.ref_nhydro.restype = c_int
    if unit in ("lmars", "hllc"):
        L.ref_riemann.restype = c_int
        L.ref_riemann.argtypes = [POINTER(Thermo), c_double, c_double, c_int, c_void_p, c_void_p,
                                  c_void_p, c_int64]
        L.ref_sound_speed.restype = c_int
        L.ref_sound_speed.argtypes = [POINTER(Thermo), c_double, c_double, c_void_p, c_void_p,
                                      c_int64]
    elif unit == "implicit":
        L.ref_implicit_correction.restype = c_int
        L.ref_implicit_correction.argtypes = [POINTER(Thermo), c_double, c_double] + \
            [c_int] * 10 + [c_void_p, c_double, c_double, c_void_p, c_void_p, c_double]
    else:
        L.ref_change_to_temperature.restype = c_int
        L.ref_change_to_temperature.argtypes = [POINTER(Thermo), c_double] + [c_int] * 5 + \
            [c_void_p, c_void_p] + [c_int] * 4 + [c_void_p] * 4
        L.ref_restore_from_temperature.restype = c_int
        L.ref_restore_from_temperature.argtypes = [POINTER(Thermo), c_double] + [c_int] * 5 + \
            [c_void_p] * 8 + [c_int] * 4
    _libs[key] = L
    return L


def _check(L, rc):
    if rc:
        raise RuntimeError(L.ref_last_error().decode())


def riemann(unit, th, mu_d, cvd_R, ivx, wl, wr):
    """The reference's Hydro::RiemannSolver (unit "lmars" or "hllc") on faces
    wl, wr (NV, n); returns flx (NV, n)."""
    wl = np.ascontiguousarray(wl, dtype=np.float64)
    wr = np.ascontiguousarray(wr, dtype=np.float64)
    flx = np.zeros_like(wl)
    L = lib(unit, wl.shape[0])
    _check(L, L.ref_riemann(ctypes.byref(th), mu_d, cvd_R, ivx, wl.ctypes.data, wr.ctypes.data,
                            flx.ctypes.data, wl.shape[1]))
    return flx


def sound_speed(th, mu_d, cvd_R, w):
    w = np.ascontiguousarray(w, dtype=np.float64)
    cs = np.zeros(w.shape[1])
    L = lib("hllc", w.shape[0])
    _check(L, L.ref_sound_speed(ctypes.byref(th), mu_d, cvd_R, w.ctypes.data, cs.ctypes.data,
                                w.shape[1]))
    return cs


def change_to_temperature(th, mu_d, is_, ie, dx1f, bc, w, kl, ku, jl, ju):
    """Decomposition::ChangeToTemperature over columns kl..ku x jl..ju of the
    block w (NV, nc3, nc2, nc1); returns (w decomposed, psf, psv, gamma)."""
    w = np.array(w, dtype=np.float64, order="C")
    nv, nc3, nc2, nc1 = w.shape
    psf = np.zeros((nc3, nc2, nc1 + 1))
    psv = np.zeros((nc3, nc2, nc1))
    gam = np.zeros((nc3, nc2, nc1))
    dx1f = np.ascontiguousarray(dx1f, dtype=np.float64)
    bc = np.ascontiguousarray(bc, dtype=np.int32)
    L = lib("decomp", nv)
    _check(L, L.ref_change_to_temperature(ctypes.byref(th), mu_d, nc3, nc2, nc1, is_, ie,
                                          dx1f.ctypes.data, bc.ctypes.data, kl, ku, jl, ju,
                                          w.ctypes.data, psf.ctypes.data, psv.ctypes.data,
                                          gam.ctypes.data))
    return w, psf, psv, gam


def restore_from_temperature(th, mu_d, is_, ie, dx1f, bc, psf, psv, gam, w, wl, wr, k, j, il, iu):
    """Decomposition::RestoreFromTemperature of column (k, j): returns
    (w, wl, wr) restored (w (NV, nc3, nc2, nc1), wl / wr (NV, nc1 + 1))."""
    w = np.array(w, dtype=np.float64, order="C")
    wl = np.array(wl, dtype=np.float64, order="C")
    wr = np.array(wr, dtype=np.float64, order="C")
    nv, nc3, nc2, nc1 = w.shape
    dx1f = np.ascontiguousarray(dx1f, dtype=np.float64)
    bc = np.ascontiguousarray(bc, dtype=np.int32)
    psf, psv, gam = (np.ascontiguousarray(a, dtype=np.float64) for a in (psf, psv, gam))
    L = lib("decomp", nv)
    _check(L, L.ref_restore_from_temperature(ctypes.byref(th), mu_d, nc3, nc2, nc1, is_, ie,
                                             dx1f.ctypes.data, bc.ctypes.data, psf.ctypes.data,
                                             psv.ctypes.data, gam.ctypes.data, w.ctypes.data,
                                             wl.ctypes.data, wr.ctypes.data, k, j, il, iu))
    return w, wl, wr


def implicit_correction(th, mu_d, cvd_R, full, w, du, dx1f, dx2, dx3, is_, ie, js, je, ks, ke,
                        dt):
    """The reference's ImplicitSolver (PartialCorrection, or FullCorrection
    when full) over the interior columns of a Cartesian block: returns du
    (NV, nc3, nc2, nc1) corrected, from the primitive state w."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    du = np.array(du, dtype=np.float64, order="C")
    nv, nc3, nc2, nc1 = w.shape
    dx1f = np.ascontiguousarray(dx1f, dtype=np.float64)
    L = lib("implicit", nv)
    _check(L, L.ref_implicit_correction(ctypes.byref(th), mu_d, cvd_R, 1 if full else 0, nc3,
                                        nc2, nc1, is_, ie, js, je, ks, ke, dx1f.ctypes.data,
                                        dx2, dx3, w.ctypes.data, du.ctypes.data, dt))
    return du
