"""Implicit solves along x2 and x3 (SolveImplicit3D X2DIR / X3DIR, canoe
src/snap/implicit/solve_implicit_3d.cpp:25-89) on the GPU against the oracle.

The GPU gathers w and du into line-major scratch by tile transposes, solves
every line with the x1 pencil kernel's cyclic reduction (periodic lines by
the bordered form) and scatters IDN, the normal momentum and IEN back; the
oracle eliminates each line sequentially as the reference does.  Both solve
the same systems, so FP64 results agree to evaluation order.
"""
import numpy as np
import pytest

from canoe_b200 import MeshBlock, problems
from canoe_b200._abi import BC_PERIODIC, BC_REFLECT, RECON_PLM, RS_LMARS
from conftest import max_var_rel_l2, rel_l2

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-11
VAR_TOL = 5e-11


def box(flag, bc=BC_PERIODIC, nx1=20, nx2=24, nx3=10, **kw):
    p = problems.periodic_x1(nx1=nx1, nx2=nx2, nx3=nx3, x1max=100.0 * nx1,
                             x2max=120.0 * nx2, x3max=90.0 * max(nx3, 1), moist=False,
                             implicit_flag=flag, **kw)
    for q in range(6):
        p.cfg.bc[q] = bc
    return p


@pytest.mark.parametrize("flag", [2, 4, 6, 7, 10, 12, 15])
@pytest.mark.parametrize("bc", [BC_PERIODIC, BC_REFLECT])
def test_line_solve_implicit(oracle_mod, flag, bc):
    p = box(flag, bc)
    gpu = MeshBlock(p)
    ora = oracle_mod.OracleBlock(p)
    rng = np.random.Generator(np.random.PCG64(17 + flag))
    du = np.zeros(p.u.shape)
    p.interior(du)[...] = 1e-3 * rng.standard_normal(p.interior(du).shape) * \
        np.abs(p.interior(p.u)).mean(axis=(1, 2, 3))[:, None, None, None]
    a = gpu.solve_implicit(du, 2.0)
    b = ora.solve_implicit(du, 2.0)
    assert max_var_rel_l2(p.interior(a), p.interior(b)) < 1e-11
    # the solves acted, and slots the reference does not copy back stayed
    assert not np.allclose(p.interior(a), p.interior(du))
    if not flag & 1:
        d = 2 if flag & 4 else 1
        for s in {1, 2, 3} - ({2} if flag & 2 else set()) - ({3} if flag & 4 else set()):
            assert np.array_equal(p.interior(a)[s], p.interior(du)[s]), s
    gpu.close()


def _steps(oracle_mod, p, nsteps=3, graph=False):
    gpu = MeshBlock(p, graph=graph)
    ora = oracle_mod.OracleBlock(p)
    dt = ora.new_dt()
    assert abs(gpu.new_dt() - dt) <= 1e-12 * dt
    for s in range(nsteps):
        ora.step(dt)
        gpu.step(dt)
        a, b = p.interior(gpu.conserved()), p.interior(ora.conserved())
        per = [rel_l2(a[n], b[n], floor=1e-12 * np.linalg.norm(b)) for n in range(b.shape[0])]
        assert rel_l2(a, b) < STEP_TOL, (s, rel_l2(a, b))
        assert max(per) < VAR_TOL, (s, per)
    assert gpu.error_word() == 0
    gpu.close()


@pytest.mark.parametrize("flag,bc,scheme", [
    (6, BC_PERIODIC, "ppm_hllc"), (7, BC_PERIODIC, "ppm_hllc"), (15, BC_PERIODIC, "ppm_hllc"),
    (7, BC_REFLECT, "plm_lmars"), (14, BC_REFLECT, "ppm_hllc"), (2, BC_PERIODIC, "plm_lmars")])
def test_line_step_parity(oracle_mod, flag, bc, scheme):
    kw = dict(recon=RECON_PLM, rsolver=RS_LMARS) if scheme == "plm_lmars" else {}
    _steps(oracle_mod, box(flag, bc, **kw))


def test_line_step_2d_and_graph(oracle_mod):
    _steps(oracle_mod, box(3, BC_PERIODIC, nx1=16, nx2=40, nx3=1))
    _steps(oracle_mod, box(7, BC_PERIODIC), graph=True)


def test_line_fp32_near_fp64():
    p64, p32 = box(7), box(7)
    p32.cfg.precision = 1  # FP32 fluxes on the perturbation
    g64, g32 = MeshBlock(p64), MeshBlock(p32)
    dt = g64.new_dt()
    for _ in range(4):
        g64.step(dt)
        g32.step(dt)
    a, b = p64.interior(g32.conserved()), p64.interior(g64.conserved())
    mom = np.linalg.norm(b[1:4])
    errs = [rel_l2(a[n], b[n], floor=(mom if 1 <= n <= 3 else 0.)) for n in range(5)]
    assert max(errs) < 1e-6, errs
    assert g32.error_word() == 0
    g64.close()
    g32.close()


def test_moist_line_solves_refused():
    p = problems.periodic_x1(nx1=8, nx2=8, nx3=4, moist=True, implicit_flag=2)
    with pytest.raises(RuntimeError, match="dry block"):
        MeshBlock(p)
