"""The device cubed-sphere shell against the oracle.

The ghost exchange is a gather with the same interpolation weights and a
precomputed 2 x 2 velocity map per ghost cell (the reference rotates each
vector through a chain of six transforms), so exchanged values agree to
1e-12 relative.  The transverse momentum flux of an x2 / x3 face is, after
FluxToGlobal and the covariant projection, the small difference of two
pressure-sized terms (the face cosine enters once from the metric table and
once recomputed), so it carries O(1e-16 p) of rounding that FMA placement
changes: fluxes are held to 1e-12 of the face's full flux vector and to
1e-10 per variable.  Steps carry the FP64 bar of the Cartesian path.
"""
import numpy as np
import pytest

from canoe_b200 import Shell, problems
from canoe_b200._abi import NGHOST as NG
from conftest import rel_l2
from test_exo3_oracle import _fields, _slabs, cell_volumes, ghost_errors

pytestmark = pytest.mark.gpu


def test_ghost_exchange_matches_oracle(oracle_mod):
    N = 16
    p, u, exact, X, Y = _fields(N)
    ora = oracle_mod.OracleShell(p)
    ora.set_conserved(u, fill=False)
    ora.fill_ghosts()
    ref = ora.conserved()
    sh = Shell(p, fill=False)
    sh.set_conserved(u, fill=False)
    sh.fill_ghosts()
    got = sh.conserved()
    for q in range(6):
        for ks, js in _slabs(N):
            a, b = got[q][:, ks, js, NG:-NG], ref[q][:, ks, js, NG:-NG]
            scale = np.abs(b).max(axis=(1, 2, 3)) + 1e-300
            scale[2:4] = scale[2:4].max()  # the momentum is one vector
            assert (np.abs(a - b) / scale[:, None, None, None]).max() < 1e-12, q
    # and the device ghosts approximate the exact fields as the oracle's do
    ef, ev = ghost_errors(got, exact, X, Y, N)
    assert ef < 5e-4 and ev < 2e-2


def _c3_small():
    return problems.shell_c3(nx1=16, nside=8, jet=5.0)


def test_primitive_matches_oracle(oracle_mod):
    p = _c3_small()
    ora = oracle_mod.OracleShell(p)
    sh = Shell(p)
    assert sh.error_word() == 0
    a, b = p.interior(sh.primitive()), p.interior(ora.primitive())
    assert rel_l2(a, b) < 1e-14


def test_fluxes_match_oracle(oracle_mod):
    p = _c3_small()
    ora = oracle_mod.OracleShell(p)
    sh = Shell(p)
    g1, g2, g3 = sh.calculate_fluxes()
    r1, r2, r3 = ora.calculate_fluxes()
    N, nx1 = p.cfg.nside, p.cfg.nx1
    i = slice(NG, NG + nx1)
    jk = slice(NG, NG + N)
    fj = slice(NG, NG + N + 1)
    a2, b2 = g2[:, :, jk, fj, i], r2[:, :, jk, fj, i]
    a3, b3 = g3[:, :, fj, jk, i], r3[:, :, fj, jk, i]
    assert rel_l2(a2, b2) < 1e-12 and rel_l2(a3, b3) < 1e-12
    for n in range(5):
        assert rel_l2(a2[:, n], b2[:, n]) < 1e-10, ("x2", n)
        assert rel_l2(a3[:, n], b3[:, n]) < 1e-10, ("x3", n)
        # x1: the hydrostatic scan sums p' = p - psv, a small difference
        assert rel_l2(g1[:, n, jk, jk, NG:NG + nx1 + 1], r1[:, n, jk, jk, NG:NG + nx1 + 1]) < 2e-11, ("x1", n)


@pytest.mark.parametrize("implicit_flag", [0, 1, 9])
def test_step_matches_oracle(oracle_mod, implicit_flag):
    p = problems.shell_c3(nx1=16, nside=8, implicit_flag=implicit_flag)
    ora = oracle_mod.OracleShell(p)
    sh = Shell(p)
    dt = 5.0
    ora.step(dt, 2)
    sh.step(dt)
    sh.step(dt)
    sh.synchronize()
    assert sh.error_word() == 0
    a, b = p.interior(sh.conserved()), p.interior(ora.conserved())
    for n in range(5):
        assert rel_l2(a[:, n], b[:, n]) < 5e-11, n
    vol = cell_volumes(p)
    m0 = sum((p.interior(p.u)[q, 0] * vol).sum() for q in range(6))
    m1 = sum((a[q, 0] * vol).sum() for q in range(6))
    assert abs(m1 - m0) / m0 < 1e-14


def _c3_pair():
    p64 = problems.shell_c3(nx1=16, nside=8)
    p32 = problems.shell_c3(nx1=16, nside=8)
    p32.cfg.precision = 1  # FP32 fluxes on the hydrostatic perturbation
    return p64, p32


def test_fp32_shell_fluxes_near_fp64():
    p64, p32 = _c3_pair()
    a = Shell(p64).calculate_fluxes()
    b = Shell(p32).calculate_fluxes()
    N, nx1 = p64.cfg.nside, p64.cfg.nx1
    i, jk, fj = slice(NG, NG + nx1), slice(NG, NG + N), slice(NG, NG + N + 1)
    sel = [(slice(None), slice(None), jk, jk, slice(NG, NG + nx1 + 1)),
           (slice(None), slice(None), jk, fj, i), (slice(None), slice(None), fj, jk, i)]
    for d in range(3):
        print("flux", d + 1, rel_l2(b[d][sel[d]], a[d][sel[d]]))
        assert rel_l2(b[d][sel[d]], a[d][sel[d]]) < 1e-5, d


def test_fp32_shell_steps_near_fp64():
    p64, p32 = _c3_pair()
    s64, s32 = Shell(p64), Shell(p32)
    for _ in range(5):
        s64.step(5.0)
        s32.step(5.0)
    s64.synchronize()
    s32.synchronize()
    assert s32.error_word() == 0
    a, b = p64.interior(s64.conserved()), p64.interior(s32.conserved())
    errs = [rel_l2(b[:, n], a[:, n]) for n in range(5)]
    print("state", errs)
    assert max(errs) < 1e-6, errs
    vol = cell_volumes(p64)
    m0 = sum((a[q, 0] * vol).sum() for q in range(6))
    m1 = sum((b[q, 0] * vol).sum() for q in range(6))
    assert abs(m1 - m0) / m0 < 1e-12
