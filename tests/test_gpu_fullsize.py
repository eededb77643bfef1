"""Size-independent properties at the benchmark sizes, where the oracle would
take too long: C2 at 128x256x256 and the C3 shell at 6 x 96^2 x 64.

- Shift invariance: C2 is periodic in x2 and x3, and every cell's arithmetic
  is the same wherever its tile or column falls, so rolling the state along
  x2 / x3 commutes with an FP64 step bit for bit (fixed dt; the FP32 path's
  reference pressure is a horizontal mean whose summation order would move).
- Conservation: total mass (dry air plus species) is conserved to FP64
  roundoff by the full step in both precisions.
- Mixed against FP64: the FP32-perturbation form stays within the error the
  bench reports after the same steps.
"""
import numpy as np
import pytest

from canoe_b200 import MeshBlock, Shell, problems
from canoe_b200._abi import FP32_PERTURBATION, FP64
from test_exo3_oracle import cell_volumes

pytestmark = pytest.mark.gpu


def _c2(prec):
    p = problems.moist3d()
    p.cfg.precision = prec
    return p


def test_c2_roll_commutes_with_step():
    p = _c2(FP64)
    b = MeshBlock(p)
    dt = b.new_dt()
    b.step(dt)
    b.step(dt)
    ref = p.interior(b.conserved())
    b.close()
    q = _c2(FP64)
    sh = (37, 101)  # (k, j)
    ui = p.interior(p.u)
    q.u[...] = 0.
    q.interior(q.u)[...] = np.roll(ui, sh, axis=(1, 2))
    b = MeshBlock(q)
    b.step(dt)
    b.step(dt)
    got = q.interior(b.conserved())
    assert b.error_word() == 0
    b.close()
    assert np.array_equal(got, np.roll(ref, sh, axis=(1, 2)))


def test_c2_mass_and_mixed_error():
    out = {}
    for name, prec in (("fp64", FP64), ("mixed", FP32_PERTURBATION)):
        p = _c2(prec)
        b = MeshBlock(p)
        u0 = p.interior(b.conserved())
        m0 = u0[:4].sum()
        dt = dt0 = out.get("dt") or b.new_dt()
        out["dt"] = dt0
        for _ in range(3):
            b.step(dt)
        u = p.interior(b.conserved())
        assert b.error_word() == 0
        assert np.isfinite(u).all()
        assert abs(u[:4].sum() - m0) / m0 < 1e-13, name
        out[name] = u
        b.close()
    a, r = out["mixed"], out["fp64"]
    mom = slice(4, 7)  # IVX..IVZ with three species slots
    for n in (0, 1, 2, 3, 7):
        scale = max(np.linalg.norm(r[n]), 1e-12 * np.linalg.norm(r))
        assert np.linalg.norm(a[n] - r[n]) / scale < 1e-9, n
    assert np.linalg.norm(a[mom] - r[mom]) / np.linalg.norm(r[mom]) < 1e-6


def test_c3_mass_and_mixed_error():
    out = {}
    for name, prec in (("fp64", FP64), ("mixed", FP32_PERTURBATION)):
        p = problems.shell_c3()
        p.cfg.precision = prec
        s = Shell(p)
        vol = cell_volumes(p)
        u0 = p.interior(s.conserved())
        m0 = sum((u0[q, 0] * vol).sum() for q in range(6))
        for _ in range(3):
            s.step(60.0)
        s.synchronize()
        u = p.interior(s.conserved())
        assert s.error_word() == 0
        m1 = sum((u[q, 0] * vol).sum() for q in range(6))
        assert abs(m1 - m0) / m0 < 1e-12, name
        out[name] = u
        s.close()
    a, r = out["mixed"], out["fp64"]
    rel = lambda x, y: np.linalg.norm(x - y) / np.linalg.norm(y)
    assert rel(a[:, 0], r[:, 0]) < 1e-9
    assert rel(a[:, 1:4], r[:, 1:4]) < 1e-6
    assert rel(a[:, 4], r[:, 4]) < 1e-9
