"""CPU checks of the oracle itself (no GPU): conservation and symmetry
properties of the restated algorithms, the MLP backprop against finite
differences, and the committed golden fixtures."""
import numpy as np
import pytest

from canoe_b200 import problems, thermo
from canoe_b200._abi import RS_HLLC, RS_LMARS
from conftest import rel_l2


def test_riemann_consistency(oracle_mod):
    """F(w, w) is the physical flux for both solvers (equal states)."""
    th = thermo.earth_moist()
    rng = np.random.Generator(np.random.PCG64(4))
    n = 200
    ny = th.ny
    w = np.zeros((5 + ny, n))
    w[0] = rng.uniform(0.5, 1.3, n)
    w[1] = rng.uniform(0, 0.02, n)
    w[1 + ny:4 + ny] = rng.uniform(-20, 20, (3, n))
    w[4 + ny] = rng.uniform(5e4, 1e5, n)
    for rs in (RS_LMARS, RS_HLLC):
        f = oracle_mod.riemann(rs, th, 1 + ny, w, w)
        rho, u = w[0], w[1 + ny]
        assert np.allclose(f[0], rho * u * (1 - w[1:1 + ny].sum(axis=0)), rtol=1e-12, atol=1e-12)
        assert np.allclose(f[1 + ny], rho * u * u + w[4 + ny], rtol=1e-12)


def test_riemann_mirror_symmetry(oracle_mod):
    """swapping sides and flipping the normal velocity flips the mass flux"""
    th = thermo.dry()
    rng = np.random.Generator(np.random.PCG64(5))
    n = 100
    wl = np.zeros((5, n)); wr = np.zeros((5, n))
    for w in (wl, wr):
        w[0] = rng.uniform(0.5, 1.3, n); w[1:4] = rng.uniform(-20, 20, (3, n))
        w[4] = rng.uniform(5e4, 1e5, n)
    for rs in (RS_LMARS, RS_HLLC):
        f = oracle_mod.riemann(rs, th, 1, wl, wr)
        ml, mr = wr.copy(), wl.copy()
        ml[1] *= -1; mr[1] *= -1
        g = oracle_mod.riemann(rs, th, 1, ml, mr)
        assert np.allclose(f[0], -g[0], rtol=1e-10, atol=1e-9)


def test_cons_prim_roundtrip(oracle_mod):
    th = thermo.earth_moist()
    p = problems.moist3d(nx1=8, nx2=4, nx3=4, x1max=2000.0, x2max=1000.0, x3max=1000.0)
    w = p.interior(p.w).reshape(p.nv, -1)
    u = oracle_mod.prim_to_cons(th, w)
    w2 = oracle_mod.cons_to_prim(th, u)
    assert rel_l2(w2, w) < 1e-14


def test_rest_state_stays_at_rest(oracle_mod):
    p = problems.bubble2d(nx1=40, nx2=24, x1max=400.0, x2max=240.0, dT=0.0)
    o = oracle_mod.OracleBlock(p)
    for _ in range(20):
        o.step()
    w = p.interior(o.primitive())
    assert np.abs(w[1:3]).max() < 1e-6


def test_implicit_solve_is_linear_in_du(oracle_mod):
    """the implicit correction solves a linear system: S(a du1 + du2) =
    a S(du1) + S(du2)"""
    p = problems.moist3d(nx1=16, nx2=4, nx3=4, x1max=2000.0, x2max=1000.0, x3max=1000.0)
    o = oracle_mod.OracleBlock(p)
    rng = np.random.Generator(np.random.PCG64(6))
    d1 = np.zeros(p.u.shape); d2 = np.zeros(p.u.shape)
    p.interior(d1)[...] = rng.standard_normal(p.interior(d1).shape) * 1e-3
    p.interior(d2)[...] = rng.standard_normal(p.interior(d2).shape) * 1e-3
    s1, s2 = o.solve_implicit(d1, 0.5), o.solve_implicit(d2, 0.5)
    s12 = o.solve_implicit(3.0 * d1 + d2, 0.5)
    assert rel_l2(p.interior(s12), p.interior(3.0 * s1 + s2)) < 1e-10


def test_satadj_conserves_and_is_idempotent(oracle_mod):
    th = thermo.earth_moist()
    from test_gpu_parity import saturated_cells
    u = saturated_cells(th, 5000, seed=8)
    u0 = u.copy()
    T1, it1, fl1 = oracle_mod.satadj(th, u)
    assert np.all((fl1 & 2) == 0)
    np.testing.assert_array_equal(u[0], u0[0])
    np.testing.assert_array_equal(u[4:], u0[4:])
    assert np.max(np.abs(u[1:4].sum(axis=0) - u0[1:4].sum(axis=0)) / u0[1:4].sum(axis=0)) < 1e-14
    u1 = u.copy()
    T2, it2, _ = oracle_mod.satadj(th, u1)
    assert np.max(np.abs(T2 - T1)) < 1e-9
    assert np.max(np.abs(u1[1:4] - u[1:4])) <= 1e-12 * np.abs(u[1:4]).max()


def test_mlp_gradient_finite_differences(oracle_mod):
    rng = np.random.Generator(np.random.PCG64(9))
    nh = 8
    npar = nh * 4 + nh + nh * nh + nh + nh + 1
    p = rng.standard_normal(npar) * 0.5
    x = rng.standard_normal((64, 4))
    y = rng.standard_normal(64)
    loss, g = oracle_mod.mlp_loss_grad(p, nh, x, y)
    h = 1e-6
    for q in rng.choice(npar, 20, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[q] += h; pm[q] -= h
        fd = (oracle_mod.mlp_loss_grad(pp, nh, x, y)[0] - oracle_mod.mlp_loss_grad(pm, nh, x, y)[0]) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(g[q]))
