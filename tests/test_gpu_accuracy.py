"""Long-run accuracy of the mixed + learned form against plain FP64.

The headline form runs reconstruction and Riemann fluxes in FP32 on the
hydrostatic perturbation and starts the saturation adjustment's Newton
iteration from the learned guess; the FP64 form is the plain method.  After
200 steps of C2's physics on a 64^3 block (16 km deep, 250 m cells) the
north star's bar holds: potential temperature and total water within 1e-4
relative L2 of the FP64 run.  Total mass (dry air plus every species) is
conserved to FP64 roundoff by both.  The state at 100 % relative humidity
condenses at the first adjustment, so that the learned start and the
adjustment's liquid / ice split are exercised along the run.
"""
import numpy as np
import pytest

from canoe_b200 import MeshBlock, learned, problems
from canoe_b200._abi import FP32_PERTURBATION, FP64
from conftest import rel_l2
from test_gpu_mixed import theta

pytestmark = pytest.mark.gpu

BAR = 1e-4
STEPS = 200


def _block(rh, prec, net=None):
    p = problems.moist3d(nx1=64, nx2=64, nx3=64, x1max=16.0e3, x2max=16.0e3, x3max=16.0e3,
                         rh=rh)
    p.cfg.precision = prec
    b = MeshBlock(p, graph=True)
    if net is not None:
        b.set_mlp(net)
    return p, b


@pytest.mark.parametrize("rh", [0.8, 1.0], ids=["rh80", "rh100"])
def test_mixed_learned_200_steps_within_bar(rh):
    net = learned.default_net()
    p, ref = _block(rh, FP64)
    _, mix = _block(rh, FP32_PERTURBATION, net)
    dt = ref.new_dt()
    ref.set_fixed_dt(dt)
    mix.set_fixed_dt(dt)
    u0 = p.interior(ref.conserved())
    m0 = u0[:4].sum()
    for _ in range(STEPS):
        ref.step()
        mix.step()
    ref.synchronize()
    mix.synchronize()
    assert ref.error_word() == 0 and mix.error_word() == 0
    th = p.cfg.thermo
    wa, wb = p.interior(ref.primitive()), p.interior(mix.primitive())
    ua, ub = p.interior(ref.conserved()), p.interior(mix.conserved())
    e_theta = rel_l2(theta(th, wb), theta(th, wa))
    e_water = rel_l2(ub[1:4].sum(axis=0), ua[1:4].sum(axis=0))
    print(f"rh {rh}: {STEPS} steps, theta {e_theta:.3e}, total water {e_water:.3e}")
    assert e_theta < BAR, e_theta
    assert e_water < BAR, e_water
    for u in (ua, ub):
        assert abs(u[:4].sum() - m0) / m0 < 1e-13
    if rh >= 1.0:
        # cells condensed during the run (liquid or ice present)
        assert (ua[2] + ua[3]).max() > 0.0
        s = mix.satadj_stats()
        assert s[0] > 0 and s[3] == 0
