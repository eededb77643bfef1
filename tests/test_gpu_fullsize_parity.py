"""The CUDA path against the oracle at the benchmark configurations' full
sizes (the oracle runs with every host thread):

- C2, 128 x 256 x 256, PPM + HLLC, implicit X1 3x3, saturation adjustment:
  one FP64 step from the seeded initial state;
- C1, 150 x 100, PLM + LMARS, no implicit solve: the full 2000 steps, each
  with the device's CFL time step (checked against the oracle's own);
- C3, the six-panel shell 6 x 96^2 x 64: two FP64 steps.

Tolerances.  One step carries the FP64 bar of the per-step parity tests:
1e-11 relative L2 of the whole state, 5e-11 per variable (the hydrostatic
decomposition's p' = p - psv is a small difference of O(1e5) numbers, and
psv's log() differs by an ulp between CUDA and the host libm).  Species are
measured against the total-water norm (condensates are zero in most cells).
The momentum of these near-hydrostatic states is the small net of the
pressure gradient and gravity, each of size rho g per unit volume: two
correct FP64 evaluations differ by roundoff of those balanced terms,
eps dt rho g per step, however small their net.  Momentum is therefore
measured against the larger of its own norm and the norm of dt rho g (the
gravity impulse of one step); against its own norm alone the first step of
a fluid at rest would compare roundoff with a momentum of almost nothing.
Over C1's 2000 steps the per-step roundoff differences are carried along by
the flow; they grow no faster than linearly in a flow that is not
turbulent, so the bar after s steps is s x the per-step bar.
"""
import os

import numpy as np
import pytest

from canoe_b200 import MeshBlock, Shell, problems
from conftest import rel_l2

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-11
VAR_TOL = 5e-11


def _per_variable(a, b, ny, dt, grav):
    """relative L2 per variable; species against the total-water norm (the
    condensates are zero in most cells), the momentum components against the
    larger of the momentum vector's norm and the gravity impulse dt rho g"""
    wn = np.linalg.norm(b[1:1 + ny].sum(axis=0)) if ny else 0.0
    rho = b[:1 + ny].sum(axis=0)
    mn = max(np.linalg.norm(b[1 + ny:4 + ny]), abs(dt * grav) * np.linalg.norm(rho))
    tot = np.linalg.norm(b)
    out = []
    for n in range(b.shape[0]):
        if 1 <= n <= ny:
            floor = wn
        elif 1 + ny <= n <= 3 + ny:
            floor = mn
        else:
            floor = 1e-12 * tot
        out.append(rel_l2(a[n], b[n], floor=floor))
    return out


@pytest.fixture(scope="module")
def ora():
    from oracle import oracle
    oracle.set_threads(os.cpu_count() or 1)
    return oracle


def test_c2_full_size_step_matches_oracle(ora):
    p = problems.moist3d()
    gpu = MeshBlock(p)
    dt = gpu.new_dt()
    ob = ora.OracleBlock(p)
    dto = ob.new_dt()
    assert abs(dt - dto) <= 1e-12 * dto, (dt, dto)
    gpu.step(dt)
    assert gpu.error_word() == 0
    a = p.interior(gpu.conserved())
    gpu.close()
    ob.step(dt)
    b = p.interior(ob.conserved())
    del ob
    tot = rel_l2(a, b)
    per = _per_variable(a, b, p.ny, dt, p.cfg.thermo.grav)
    print("C2 full size, one step: state", tot, "per variable", per)
    assert tot < STEP_TOL, tot
    assert max(per) < VAR_TOL, per


def test_c1_2000_steps_match_oracle(ora):
    p = problems.bubble2d()
    assert (p.cfg.nx1, p.cfg.nx2, p.cfg.nx3) == (150, 100, 1)
    gpu = MeshBlock(p)
    ob = ora.OracleBlock(p)
    nsteps = 2000
    worst_dt = 0.0
    checkpoints = {1, 10, 100, 1000, nsteps}
    for s in range(1, nsteps + 1):
        dt = gpu.new_dt()
        dto = ob.new_dt()
        worst_dt = max(worst_dt, abs(dt - dto) / dto)
        gpu.step(dt)
        ob.step(dt)
        if s in checkpoints:
            a, b = p.interior(gpu.conserved()), p.interior(ob.conserved())
            tot = rel_l2(a, b)
            per = _per_variable(a, b, 0, dt, p.cfg.thermo.grav)
            print(f"C1 step {s}: dt {dt:.6e} state {tot:.3e} per variable "
                  + " ".join(f"{x:.2e}" for x in per))
            assert tot < STEP_TOL * s, (s, tot)
            assert max(per) < VAR_TOL * s, (s, per)
    assert gpu.error_word() == 0
    # the two CFL time steps agree throughout
    assert worst_dt < 1e-11, worst_dt
    # the bubble has risen: the state moved well beyond roundoff
    v = p.interior(gpu.conserved())[2]
    assert np.abs(v).max() > 1e-3
    gpu.close()


def test_c3_full_size_shell_two_steps_match_oracle(ora):
    p = problems.shell_c3()
    assert (p.cfg.nside, p.cfg.nx1) == (96, 64)
    sh = Shell(p)
    os_ = ora.OracleShell(p)
    dt = 60.0
    sh.step(dt)
    sh.step(dt)
    sh.synchronize()
    assert sh.error_word() == 0
    a = p.interior(sh.conserved())
    sh.close()
    os_.step(dt, 2)
    b = p.interior(os_.conserved())
    errs = [rel_l2(a[:, n], b[:, n]) for n in range(5)]
    mom = rel_l2(a[:, 1:4], b[:, 1:4])
    print("C3 full size, two steps: per variable", errs, "momentum vector", mom)
    assert rel_l2(a, b) < STEP_TOL
    assert max(errs[0], errs[4], mom) < VAR_TOL, (errs, mom)
