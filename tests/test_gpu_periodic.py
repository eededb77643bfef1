"""Periodic x1: the cyclic implicit solve of the x1 pencil kernel against the
oracle's restatement of PeriodicForwardSweep / PeriodicBackwardSubstitution
(canoe src/snap/implicit/periodic_forward_backward.hpp:15-234).

The GPU solves the cyclic system by bordering inside the block cyclic
reduction; the oracle eliminates sequentially as the reference does.  Both
solve the same system, so FP64 results agree to evaluation order: the
operator to 1e-11 relative L2 per variable, full steps to the FP64 step bar
of the non-periodic parity tests.
"""
import numpy as np
import pytest

from canoe_b200 import MeshBlock, problems
from canoe_b200._abi import BC_REFLECT, RECON_PLM, RS_LMARS
from conftest import max_var_rel_l2, rel_l2

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-11
VAR_TOL = 5e-11
FP32_PERTURBATION = 1


def case(flag, moist, **kw):
    return problems.periodic_x1(nx1=40, nx2=8, nx3=6, x1max=4000.0, moist=moist,
                                implicit_flag=flag, **kw)


@pytest.mark.parametrize("flag", [1, 9])
@pytest.mark.parametrize("moist", [False, True])
def test_periodic_solve_implicit(oracle_mod, flag, moist):
    p = case(flag, moist)
    gpu = MeshBlock(p)
    ora = oracle_mod.OracleBlock(p)
    rng = np.random.Generator(np.random.PCG64(11))
    du = np.zeros(p.u.shape)
    p.interior(du)[...] = 1e-3 * rng.standard_normal(p.interior(du).shape) * \
        np.abs(p.interior(p.u)).mean(axis=(1, 2, 3))[:, None, None, None]
    dt = 2.0
    a = gpu.solve_implicit(du, dt)
    b = ora.solve_implicit(du, dt)
    assert max_var_rel_l2(p.interior(a), p.interior(b)) < 1e-11
    if moist:
        # the periodic update keeps du of the species as it was
        ny = p.ny
        assert np.array_equal(p.interior(a)[1:1 + ny], p.interior(du)[1:1 + ny])
    gpu.close()


@pytest.mark.parametrize("flag,moist,scheme", [
    (1, False, "ppm_hllc"), (9, False, "ppm_hllc"), (1, True, "ppm_hllc"),
    (9, True, "plm_lmars"), (1, False, "plm_lmars")])
def test_periodic_step_parity(oracle_mod, flag, moist, scheme):
    kw = dict(recon=RECON_PLM, rsolver=RS_LMARS) if scheme == "plm_lmars" else {}
    p = case(flag, moist, **kw)
    gpu = MeshBlock(p)
    ora = oracle_mod.OracleBlock(p)
    dt = ora.new_dt()
    assert abs(gpu.new_dt() - dt) <= 1e-12 * dt
    for s in range(3):
        ora.step(dt)
        gpu.step(dt)
        a, b = p.interior(gpu.conserved()), p.interior(ora.conserved())
        ny = p.ny
        wn = np.linalg.norm(b[1:1 + ny].sum(axis=0)) if ny else 0.
        per = [rel_l2(a[n], b[n], floor=(wn if 1 <= n <= ny else 1e-12 * np.linalg.norm(b)))
               for n in range(b.shape[0])]
        assert rel_l2(a, b) < STEP_TOL, (s, rel_l2(a, b))
        assert max(per) < VAR_TOL, (s, per)
    assert gpu.error_word() == 0
    gpu.close()


def test_periodic_fp32_near_fp64():
    p64, p32 = case(1, True), case(1, True)
    p32.cfg.precision = FP32_PERTURBATION
    g64, g32 = MeshBlock(p64), MeshBlock(p32)
    dt = g64.new_dt()
    for _ in range(4):
        g64.step(dt)
        g32.step(dt)
    a, b = p64.interior(g32.conserved()), p64.interior(g64.conserved())
    # momentum components against the norm of the momentum vector: the
    # transverse components are 2 % of the x1 one
    ny = p64.ny
    mom = np.linalg.norm(b[1 + ny:4 + ny])
    errs = [rel_l2(a[n], b[n], floor=(mom if 1 + ny <= n <= 3 + ny else 0.))
            for n in range(b.shape[0]) if np.any(b[n])]
    assert max(errs) < 1e-6, errs
    assert g32.error_word() == 0
    g64.close()
    g32.close()


def test_periodic_rejects_one_sided_x1():
    p = case(1, False)
    p.cfg.bc[1] = BC_REFLECT
    blk = MeshBlock(p)
    with pytest.raises(RuntimeError, match="both x1 boundaries"):
        blk.step(1.0)
    blk.close()
