"""The oracle pinned to the reference's own code.

oracle/_ref holds the reference's src/snap/riemann/lmars.cpp,
src/snap/riemann/hllc_transform.cpp (Cartesian branch),
src/snap/eos/ideal_moist_hydro.cpp (SoundSpeed), src/interface/eos.hpp
(get_gamma, get_rd, get_gammad) and
src/snap/decomposition/change_to_temperature.cpp and
src/snap/implicit/{partial,full}_correction.cpp (with forward_backward.hpp
and flux_decomposition.hpp), compiled as they lie against shim headers
(oracle/ref_shim) for the libraries they include.  These tests hold the
oracle's restatement to that code on seeded inputs: the Riemann fluxes of
dry and moist face states in all three directions, the hydrostatic
decomposition of whole C1- and C2-like blocks under every x1 boundary
pairing and its inverse on the face states, and the implicit vertical
correction (3x3 and 5x5 block rows, Thomas sweep, species correction).

Tolerance: both sides are compiled by the same g++ with the same
floating-point flags (no FMA contraction) and evaluate the same formulas;
where the oracle groups a product or a half-sum differently the results
differ in the last bit.  The bar is 1e-15 of each variable's largest
magnitude (a few ulp): measured differences are about 1.2e-16 of it, and a
change of formula or constant moves results by far more (the planted-error
test below shows a 1e-9 change of gamma_d failing the pin).
"""
import numpy as np
import pytest

from canoe_b200 import problems, thermo
from canoe_b200._abi import (BC_OUTFLOW, BC_PERIODIC, BC_REFLECT, NGHOST, RS_HLLC, RS_LMARS)
from oracle import oracle, ref

pytestmark = pytest.mark.skipif(not ref.available(),
                                reason="reference source tree absent and oracle/_ref not built")

REL = 1e-15


def _close(a, b, rel=REL):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.maximum(np.abs(b), np.finfo(float).tiny)
    err = np.max(np.abs(a - b) / scale) if a.size else 0.0
    # values that are zero on both sides, or cancel to roundoff of the
    # variable's magnitude, compare against the variable's norm
    norm = np.max(np.abs(b)) if b.size else 1.0
    err_abs = np.max(np.abs(a - b)) / max(norm, np.finfo(float).tiny) if a.size else 0.0
    return min(err, err_abs) <= rel or np.array_equal(a, b), (float(err), float(err_abs))


def _faces(th, n, seed, jump):
    """Seeded primitive face states (NV, n): density, mass fractions,
    velocities and pressure of an atmosphere, the right state a jump of
    relative size `jump` away from the left one."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nv = 5 + th.ny
    wl = np.zeros((nv, n))
    wl[0] = rng.uniform(0.2, 1.4, n)
    if th.ny:
        wl[1] = rng.uniform(0.0, 0.02, n)
        for s in range(2, th.ny + 1):
            wl[s] = rng.uniform(0.0, 0.003, n)
    for v in range(3):
        wl[1 + th.ny + v] = rng.uniform(-40.0, 40.0, n)
    wl[4 + th.ny] = rng.uniform(1.0e4, 1.1e5, n)
    wr = wl * (1.0 + jump * rng.uniform(-1.0, 1.0, wl.shape))
    for v in range(3):
        wr[1 + th.ny + v] = wl[1 + th.ny + v] + 60.0 * jump * rng.uniform(-1.0, 1.0, n)
    return wl, wr


def _thermos():
    return [("dry", thermo.dry(), thermo.MU_EARTH_DRY),
            ("moist", thermo.earth_moist(), thermo.MU_EARTH_DRY)]


@pytest.mark.parametrize("rs,unit", [(RS_LMARS, "lmars"), (RS_HLLC, "hllc")])
@pytest.mark.parametrize("name,th,mu", _thermos(), ids=[t[0] for t in _thermos()])
@pytest.mark.parametrize("jump", [1e-3, 0.2, 0.9])
def test_riemann_matches_reference(rs, unit, name, th, mu, jump):
    cvd_R = 1.0 / (th.gammad - 1.0)
    assert (cvd_R + 1.0) / cvd_R == th.gammad  # get_gammad reproduces gamma_d
    wl, wr = _faces(th, 4096, seed=11 + rs, jump=jump)
    for d in range(3):
        ivx = 1 + th.ny + d
        fo = oracle.riemann(rs, th, ivx, wl, wr)
        fr = ref.riemann(unit, th, mu, cvd_R, ivx, wl, wr)
        for n in range(fo.shape[0]):
            ok, err = _close(fo[n], fr[n])
            assert ok, (unit, name, d, n, err)


@pytest.mark.parametrize("name,th,mu", _thermos(), ids=[t[0] for t in _thermos()])
def test_sound_speed_matches_reference(name, th, mu):
    """EquationOfState::SoundSpeed (ideal_moist_hydro.cpp:87-91) through
    get_gamma against the gamma the oracle uses."""
    cvd_R = 1.0 / (th.gammad - 1.0)
    w, _ = _faces(th, 2048, seed=5, jump=0.0)
    cs = ref.sound_speed(th, mu, cvd_R, w)
    ipr = 4 + th.ny
    gam = np.array([1.0 + (th.gammad - 1.0) * _feps(th, w[:, c]) / _fsig(th, w[:, c])
                    for c in range(w.shape[1])])
    np.testing.assert_allclose(cs, np.sqrt(gam * w[ipr] / w[0]), rtol=4e-16, atol=0)


def _fsig(th, w):
    f = 1.0
    for n in range(1, th.ny + 1):
        f += w[n] * th.cv_ratio_m1[n - 1]
    return f


def _feps(th, w):
    f = 1.0
    for n in range(1, th.nvapor + 1):
        f += w[n] * th.inv_mu_ratio_m1[n - 1]
    for n in range(th.nvapor + 1, th.ny + 1):
        f -= w[n]
    return f


def _blocks():
    def c1():
        return problems.bubble2d(nx1=40, nx2=12, x1max=400.0, x2max=120.0)

    def c2():
        return problems.moist3d(nx1=24, nx2=6, nx3=5, x1max=3000.0, x2max=1500.0,
                                x3max=1250.0, noise=0.5)

    return [("c1", c1, thermo.MU_EARTH_DRY), ("c2", c2, thermo.MU_EARTH_DRY)]


BCS = [(BC_REFLECT, BC_REFLECT), (BC_OUTFLOW, BC_OUTFLOW), (BC_REFLECT, BC_OUTFLOW),
       (BC_PERIODIC, BC_PERIODIC)]


@pytest.mark.parametrize("bc", BCS, ids=["reflect", "outflow", "reflect-outflow", "periodic"])
@pytest.mark.parametrize("name,make,mu", _blocks(), ids=[b[0] for b in _blocks()])
def test_decomposition_matches_reference(bc, name, make, mu):
    """ChangeToTemperature over all interior columns, then
    RestoreFromTemperature of every column's face states, against the
    oracle's column functions."""
    p = make()
    p.cfg.bc[0], p.cfg.bc[1] = bc
    ob = oracle.OracleBlock(p)
    # a perturbed state so that every column differs
    rng = np.random.Generator(np.random.PCG64(3))
    w = ob.primitive()
    w *= 1.0 + 1e-3 * rng.uniform(-1.0, 1.0, w.shape)
    ob.set_primitive(w)
    th = p.cfg.thermo
    nv, nc3, nc2, nc1 = w.shape
    is_, ie = NGHOST, NGHOST + p.cfg.nx1 - 1
    ks, ke = (NGHOST, NGHOST + p.cfg.nx3 - 1) if p.cfg.nx3 > 1 else (0, 0)
    js, je = (NGHOST, NGHOST + p.cfg.nx2 - 1) if p.cfg.nx2 > 1 else (0, 0)
    x1f = np.zeros(nc1 + 1)
    x1f[is_:ie + 2] = p.x1f
    for g in range(1, NGHOST + 1):
        x1f[is_ - g] = 2 * x1f[is_] - x1f[is_ + g]
        x1f[ie + 1 + g] = 2 * x1f[ie + 1] - x1f[ie + 1 - g]
    dx1f = np.diff(x1f)
    bc6 = [p.cfg.bc[q] for q in range(6)]
    wref, psf, psv, gam = ref.change_to_temperature(th, mu, is_, ie, dx1f, bc6, w, ks, ke, js, je)
    assert np.isfinite(psf[ks:ke + 1, js:je + 1]).all()
    ipr = 4 + th.ny
    for k in range(ks, ke + 1):
        for j in range(js, je + 1):
            q, pf, pv, gm = ob.x1_change_to_temperature(k, j)
            for a, b, what in ((q, wref[:, k, j], "w"), (pf, psf[k, j], "psf"),
                               (pv, psv[k, j], "psv"), (gm, gam[k, j], "gamma")):
                ok, err = _close(a, b)
                assert ok, (name, bc, k, j, what, err)
            # face states of the decomposed pencil (first order plus noise),
            # a few with p' far below -psf to reach the pressure floor
            wl = np.zeros((nv, nc1 + 1))
            wr = np.zeros((nv, nc1 + 1))
            wl[:, 1:] = q
            wr[:, :-1] = q
            wl *= 1.0 + 1e-4 * rng.uniform(-1, 1, wl.shape)
            wr *= 1.0 + 1e-4 * rng.uniform(-1, 1, wr.shape)
            wl[ipr, is_ + 2] = -3.0 * pf[is_ + 2]
            wr[ipr, ie - 1] = -3.0 * pf[ie - 1]
            qo, lo, ro = ob.x1_restore_from_temperature(k, j, q, wl, wr, is_, ie + 1)
            wfull = wref.copy()
            wr2, lr, rr = ref.restore_from_temperature(th, mu, is_, ie, dx1f, bc6, psf, psv, gam,
                                                       wfull, wl, wr, k, j, is_, ie + 1)
            for a, b, what in ((qo, wr2[:, k, j], "w"), (lo[:, is_:ie + 2], lr[:, is_:ie + 2], "wl"),
                               (ro[:, is_:ie + 2], rr[:, is_:ie + 2], "wr")):
                ok, err = _close(a, b)
                assert ok, (name, bc, k, j, what, err)


def test_pin_detects_a_planted_error():
    """The comparison is sensitive: the oracle run with gamma_d off by 1e-9
    (a planted mistake in the oracle's input) no longer matches the
    reference."""
    th = thermo.earth_moist()
    cvd_R = 1.0 / (th.gammad - 1.0)
    wl, wr = _faces(th, 1024, seed=2, jump=0.2)
    ivx = 1 + th.ny
    fr = ref.riemann("hllc", th, thermo.MU_EARTH_DRY, cvd_R, ivx, wl, wr)
    bad = thermo.earth_moist()
    bad.gammad = th.gammad * (1.0 + 1e-9)
    fo = oracle.riemann(RS_HLLC, bad, ivx, wl, wr)
    assert not all(_close(fo[n], fr[n])[0] for n in range(fo.shape[0]))


@pytest.mark.parametrize("flag", [1, 9], ids=["partial3x3", "full5x5"])
@pytest.mark.parametrize("name,make,mu", _blocks(), ids=[b[0] for b in _blocks()])
def test_implicit_correction_matches_reference(flag, name, make, mu):
    """ImplicitSolver::PartialCorrection / FullCorrection (the reference's
    Eigen code, inverses from the shim) against the oracle's block solve on
    a perturbed state and a seeded du.  Tolerance, relative L2 per variable:
    the two sides form the same block rows and eliminate in the same
    (Thomas) order; they differ in how each block inverse is evaluated.  The
    3x3 inverses are both adjugates (measured <= 5e-16: 1e-14); the 5x5 ones
    Gauss-Jordan with partial pivoting, whose roundoff the blocks' spread of
    scale (1/dt against c^2 rho terms) amplifies (measured <= 1e-11:
    1e-10)."""
    p = make()
    p.cfg.implicit_flag = flag
    ob = oracle.OracleBlock(p)
    rng = np.random.Generator(np.random.PCG64(11))
    w = ob.primitive()
    w *= 1.0 + 1e-3 * rng.uniform(-1.0, 1.0, w.shape)
    ob.set_primitive(w)
    th = p.cfg.thermo
    nv, nc3, nc2, nc1 = w.shape
    du = np.zeros(w.shape)
    p.interior(du)[...] = 1e-3 * rng.standard_normal(p.interior(du).shape) * \
        np.abs(p.interior(p.u)).mean(axis=(1, 2, 3))[:, None, None, None]
    dt = 0.3
    got = ob.solve_implicit(du, dt)
    is_, ie = NGHOST, NGHOST + p.cfg.nx1 - 1
    ks, ke = (NGHOST, NGHOST + p.cfg.nx3 - 1) if p.cfg.nx3 > 1 else (0, 0)
    js, je = (NGHOST, NGHOST + p.cfg.nx2 - 1) if p.cfg.nx2 > 1 else (0, 0)
    x1f = np.zeros(nc1 + 1)
    x1f[is_:ie + 2] = p.x1f
    for g in range(1, NGHOST + 1):
        x1f[is_ - g] = 2 * x1f[is_] - x1f[is_ + g]
        x1f[ie + 1 + g] = 2 * x1f[ie + 1] - x1f[ie + 1 - g]
    ref_du = ref.implicit_correction(th, mu, 1.0 / (th.gammad - 1.0), flag & 8, w, du,
                                     np.diff(x1f), p.cfg.dx2, p.cfg.dx3, is_, ie, js, je, ks,
                                     ke, dt)
    a, b = p.interior(got), p.interior(ref_du)
    tol = 1e-14 if flag == 1 else 1e-10
    top = max(np.linalg.norm(b[n]) for n in range(nv))
    for n in range(nv):
        err = np.linalg.norm(a[n] - b[n]) / max(np.linalg.norm(b[n]), 1e-12 * top)
        assert err < tol, (name, flag, n, err)
    # and the correction did change du
    assert np.linalg.norm(p.interior(ref_du - du)) > 1e-6 * np.linalg.norm(p.interior(du))
