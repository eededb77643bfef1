"""The oracle's cubed-sphere exchange against analytic fields (CPU).

The reference ships no outputs for its exo3 path, so the restated exchange
(PackData / InteprolateX2, X3 / TransformOX unpacked in standard order) is
pinned against geometry instead: a smooth scalar and a solid-body zonal
wind are set in every panel's interior, the ghosts are exchanged, and each
ghost value is compared with the exact field at the ghost cell's own
position.  The errors must shrink at second order with the panel size: a
wrong orientation, reversal or rotation anywhere on the 24 panel edges
gives O(1) errors instead.
"""
import numpy as np
import pytest

from canoe_b200 import cubed_sphere as cs
from canoe_b200 import problems
from canoe_b200._abi import NGHOST as NG


def _fields(N, nx1=4):
    p = problems.shell_c3(nx1=nx1, nside=N)
    _, av = cs.panel_angles(N)
    n = N + 2 * NG
    u = np.zeros((6, 5, n, n, nx1 + 2 * NG))
    X, Y = np.broadcast_arrays(np.tan(av)[None, :], np.tan(av)[:, None])  # (k, j)
    ing = slice(NG, NG + N)
    exact = []
    for q in range(6):
        b = q + 1
        r = cs.xyz(b, X, Y)
        f = 1.0 + 0.1 * r[0] + 0.2 * r[1] + 0.3 * r[2]
        lat, _ = cs.latlon(b, X, Y)
        U = 10.0 * np.cos(lat)
        v2, v3 = cs.velocity_from_uv(b, X, Y, U, np.zeros_like(U))
        cth = cs.cos_theta(X, Y)
        exact.append((f, U))
        u[q, 0, ing, ing, :] = f[ing, ing][:, :, None]
        u[q, 2, ing, ing, :] = (v2 + v3 * cth)[ing, ing][:, :, None]
        u[q, 3, ing, ing, :] = (v3 + v2 * cth)[ing, ing][:, :, None]
        u[q, 4, ing, ing, :] = 1.0e5
    return p, u, exact, X, Y


def _slabs(N):
    a, b, c = slice(NG, NG + N), slice(0, NG), slice(NG + N, 2 * NG + N)
    return [(a, b), (a, c), (b, a), (c, a)]


def ghost_errors(ug, exact, X, Y, N):
    """max scalar and wind errors over all ghost slabs"""
    ef = ev = 0.0
    for q in range(6):
        f, U = exact[q]
        for ks, js in _slabs(N):
            ef = max(ef, np.abs(ug[q, 0, ks, js, NG] - f[ks, js]).max())
            x, y = X[ks, js], Y[ks, js]
            cth = cs.cos_theta(x, y)
            s2 = 1 - cth ** 2
            m2, m3 = ug[q, 2, ks, js, NG], ug[q, 3, ks, js, NG]
            v2, v3 = m2 / s2 - m3 * cth / s2, -m2 * cth / s2 + m3 / s2
            Ug, Vg = cs.uv_from_velocity(q + 1, x, y, v2, v3)
            ev = max(ev, np.abs(Ug - U[ks, js]).max(), np.abs(Vg).max())
    return ef, ev


def test_exchange_second_order(oracle_mod):
    errs = []
    for N in (8, 16, 32):
        p, u, exact, X, Y = _fields(N)
        s = oracle_mod.OracleShell(p)
        s.set_conserved(u, fill=False)
        s.fill_ghosts()
        errs.append(ghost_errors(s.conserved(), exact, X, Y, N))
    (f8, v8), (f16, v16), (f32, v32) = errs
    # the fields vary by O(0.4) and O(10 m/s) over the sphere
    assert f32 < 2e-4 and v32 < 5e-3, errs
    for a, b in ((f8, f16), (f16, f32), (v8, v16), (v16, v32)):
        assert 3.0 < a / b < 5.0, errs  # second order: ratio ~4 per halving


def test_shell_step_conserves_mass(oracle_mod):
    """the L/R swap makes both panels of an edge use one pair of states, so
    the shell conserves total mass to roundoff"""
    p = problems.shell_c3(nx1=8, nside=8)
    s = oracle_mod.OracleShell(p)
    vol = cell_volumes(p)

    def mass():
        return sum((p.interior(s.conserved())[q, 0] * vol).sum() for q in range(6))

    m0 = mass()
    s.step(5.0, 2)
    w = p.interior(s.primitive())
    assert np.isfinite(w).all()
    assert abs(mass() - m0) / m0 < 1e-14


def cell_volumes(p):
    """GnomonicEquiangle::CellVolume of the interior cells of one panel"""
    N, x1f = p.cfg.nside, p.x1f
    xf, xv = cs.panel_angles(N)
    ing = slice(NG, NG + N)
    x, y = np.tan(xv[ing])[None, :], np.tan(xv[ing])[:, None]
    x1, x2 = np.tan(xf[NG:NG + N])[None, :], np.tan(xf[NG + 1:NG + N + 1])[None, :]
    y1, y2 = np.tan(xf[NG:NG + N])[:, None], np.tan(xf[NG + 1:NG + N + 1])[:, None]
    a2 = np.arccos((1 + x1 * x2 + y * y) / (np.sqrt(1 + x1 ** 2 + y * y) * np.sqrt(1 + x2 ** 2 + y * y)))
    a3 = np.arccos((1 + x * x + y1 * y2) / (np.sqrt(1 + x * x + y1 ** 2) * np.sqrt(1 + x * x + y2 ** 2)))
    sinc = np.sqrt(1 + x * x + y * y) / (np.sqrt(1 + x * x) * np.sqrt(1 + y * y))
    x1v = 0.5 * (x1f[1:] + x1f[:-1])
    return (a2 * a3 * sinc)[:, :, None] * (x1v ** 2 * np.diff(x1f))[None, None, :]
