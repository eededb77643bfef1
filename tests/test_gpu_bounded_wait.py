"""The bounded waits that guard the kernels' bulk copies give up with an
error bit instead of hanging: a wait for an mbarrier phase that cannot
complete reports CANOE_EBIT_TIMEOUT after its spin limit, a wait for a
completed phase reports nothing, and the device stays usable afterwards."""
import ctypes

import numpy as np
import pytest

from canoe_b200 import MeshBlock, problems
from canoe_b200._abi import check, load

pytestmark = pytest.mark.gpu

CANOE_EBIT_TIMEOUT = 32


def _wait(spins, complete):
    bits = ctypes.c_uint32(0xFFFF)
    check(load().canoe_selftest_bounded_wait(spins, complete, ctypes.byref(bits)),
          "canoe_selftest_bounded_wait")
    return bits.value


def test_wait_that_cannot_complete_times_out():
    assert _wait(1000, 0) == CANOE_EBIT_TIMEOUT


def test_completed_phase_does_not_time_out():
    assert _wait(1000, 1) == 0


def test_device_usable_after_timeout():
    assert _wait(200, 0) == CANOE_EBIT_TIMEOUT
    p = problems.bubble2d(nx1=40, nx2=24, x1max=400.0, x2max=240.0)
    b = MeshBlock(p)
    b.step(0.05)
    assert b.error_word() == 0
    assert np.isfinite(b.conserved()).all()
    b.close()


def test_rejects_bad_arguments():
    bits = ctypes.c_uint32(0)
    assert load().canoe_selftest_bounded_wait(0, 0, ctypes.byref(bits)) != 0
    assert load().canoe_selftest_bounded_wait(10, 0, None) != 0


def _umma_wait(spins, issue):
    bits = ctypes.c_uint32(0xFFFF)
    check(load().canoe_selftest_umma_wait(spins, issue, ctypes.byref(bits)),
          "canoe_selftest_umma_wait")
    return bits.value


def test_tensor_core_wait_without_mmas_times_out():
    """No MMA is issued, so the completion wait of the warm-start inference
    cannot succeed: it reports the timeout and frees its tensor memory."""
    assert _umma_wait(1000, 0) == CANOE_EBIT_TIMEOUT


def test_tensor_core_wait_with_mmas_completes():
    """Committed MMAs on zero operands complete within the bound and leave a
    zero accumulator."""
    assert _umma_wait(1 << 18, 1) == 0


def test_device_usable_after_tensor_core_timeout():
    """After a timed-out wait (tensor memory freed), the tensor-core
    inference still runs and gives finite outputs."""
    from canoe_b200 import learned
    assert _umma_wait(200, 0) == CANOE_EBIT_TIMEOUT
    net = learned.WarmStartNet(seed=3)
    x = np.random.default_rng(0).standard_normal((3000, 4)).astype(np.float32)
    y = net.forward(x, tensor_core=True)
    assert np.isfinite(y).all()
    assert _umma_wait(1 << 18, 1) == 0
