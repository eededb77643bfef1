"""The FP32-on-perturbation flux path against the FP64 path.

Reconstruction and Riemann fluxes run in FP32 on p' = p - p_ref with an FP64
hydrostatic reference; the divergence, implicit solve, RK registers and the
saturation adjustment stay FP64.  Stated errors (relative L2 against FP64):
fluxes <= 1e-5 per variable; potential temperature and total water after
20 steps <= 1e-6; total mass conserved to FP64 roundoff.
"""
import numpy as np
import pytest

from canoe_b200 import MeshBlock, problems, thermo
from canoe_b200._abi import FP32_PERTURBATION, RECON_PLM, RS_LMARS
from conftest import rel_l2
from test_gpu_parity import perturb, small_c1, small_c2

pytestmark = pytest.mark.gpu


def fp32(p):
    p.cfg.precision = FP32_PERTURBATION
    return p


def theta(th, w, p0=1.0e5):
    """potential temperature of a primitive state (dry exponent)"""
    ny = th.ny
    q = w[1:1 + ny]
    feps = thermo.feps_of(th, q) if ny else 1.0
    T = w[4 + ny] / (w[0] * th.rd * feps)
    kappa = (th.gammad - 1.0) / th.gammad
    return T * (p0 / w[4 + ny]) ** kappa


@pytest.mark.parametrize("case", ["c1", "c2", "c2_plm_lmars"])
def test_fp32_fluxes_close_to_fp64(oracle_mod, case):
    mk = {"c1": lambda: small_c1(),
          "c2": lambda: small_c2(),
          "c2_plm_lmars": lambda: small_c2(recon=RECON_PLM, rsolver=RS_LMARS)}[case]
    p = perturb(mk())
    ora = oracle_mod.OracleBlock(p)
    ref = ora.calculate_fluxes()
    got = MeshBlock(fp32(p)).calculate_fluxes()
    for d in range(3 if p.cfg.nx3 > 1 else 2):
        a, b = got[d], ref[d]
        top = max(np.linalg.norm(b[n]) for n in range(b.shape[0]))
        for n in range(b.shape[0]):
            err = rel_l2(a[n], b[n], floor=1e-6 * top)
            assert err < 1e-5, f"x{d + 1} var {n}: {err}"


def test_fp32_steps_theta_and_water(oracle_mod):
    p = perturb(small_c2(nx1=32, nx2=24, nx3=24, x1max=4000.0, x2max=6000.0, x3max=6000.0),
                dv=1.0)
    a = MeshBlock(p)
    b = MeshBlock(fp32(problems.moist3d(nx1=32, nx2=24, nx3=24, x1max=4000.0,
                                        x2max=6000.0, x3max=6000.0)))
    b.set_conserved(p.u)
    dt = a.new_dt()
    u0 = p.interior(b.conserved())
    m0 = u0[:4].sum()
    for _ in range(20):
        a.step(dt)
        b.step(dt)
    th = p.cfg.thermo
    wa, wb = p.interior(a.primitive()), p.interior(b.primitive())
    ua, ub = p.interior(a.conserved()), p.interior(b.conserved())
    e_theta = rel_l2(theta(th, wb), theta(th, wa))
    e_water = rel_l2(ub[1:4].sum(axis=0), ua[1:4].sum(axis=0))
    assert e_theta < 1e-6, e_theta
    assert e_water < 1e-6, e_water
    assert abs(ub[:4].sum() - m0) / m0 < 1e-13
    assert b.error_word() == 0


def test_fp32_dry_bubble_runs():
    p = perturb(small_c1(), dv=0.5)
    a = MeshBlock(p)
    b = MeshBlock(fp32(small_c1()))
    b.set_conserved(p.u)
    for _ in range(10):
        dt = a.new_dt()
        a.step(dt)
        b.step(dt)
    ua, ub = p.interior(a.conserved()), p.interior(b.conserved())
    assert rel_l2(ub[4], ua[4]) < 1e-8  # total energy
    assert rel_l2(ub[0], ua[0]) < 1e-8  # density
