"""canoe_block_step_noalloc against canoe_block_step.

The no-allocation step launches the same kernels as the block step with its
scratch in a fixed device array, so two calls in a row must give the same
bits as two block steps with the same dt.  The file name sorts last so that
the test also runs after every other test of the session has used the
device.
"""
import ctypes

import numpy as np
import pytest

from canoe_b200 import MeshBlock, problems
from canoe_b200._abi import RECON_PLM, RS_LMARS, check, load

pytestmark = pytest.mark.gpu

FP32_PERTURBATION = 1
CANOE_ERR_ARG = 1
CANOE_ERR_UNSUPPORTED = 5


def _noalloc_two_steps(p, dt):
    import torch
    lib = load()
    u = torch.from_numpy(np.ascontiguousarray(p.u)).cuda()
    w = torch.zeros_like(u)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    torch.cuda.synchronize()
    out = []
    for _ in range(2):
        check(lib.canoe_block_step_noalloc(ctypes.byref(p.cfg), u.data_ptr(), w.data_ptr(),
                                           err.data_ptr(), float(dt), ctypes.c_void_p(s.cuda_stream)),
              "canoe_block_step_noalloc")
        s.synchronize()
        out.append((u.cpu().numpy(), w.cpu().numpy(), int(err.item())))
    return out


def _block_two_steps(p, dt, reset_profile):
    blk = MeshBlock(p)
    out = []
    for _ in range(2):
        if reset_profile:
            # the FP32 path's pressure profile is that of the state on entry
            blk.set_conserved(blk.conserved())
        blk.step(dt)
        out.append((blk.conserved(), blk.primitive(), blk.error_word()))
    blk.close()
    return out


def _cases():
    return [
        ("moist3d-fp64", lambda: problems.moist3d(nx1=24, nx2=16, nx3=12, x1max=3000.0,
                                                  x2max=4000.0, x3max=3000.0, noise=0.5)),
        ("moist3d-fp32", lambda: problems.moist3d(nx1=24, nx2=16, nx3=12, x1max=3000.0,
                                                  x2max=4000.0, x3max=3000.0, noise=0.5)),
        ("bubble2d-plm-lmars", lambda: problems.bubble2d(nx1=40, nx2=24, x1max=400.0,
                                                         x2max=240.0, recon=RECON_PLM,
                                                         rsolver=RS_LMARS)),
    ]


@pytest.mark.parametrize("name,make", _cases(), ids=[c[0] for c in _cases()])
def test_noalloc_matches_block_step(name, make):
    p = make()
    if name.endswith("fp32"):
        p.cfg.precision = FP32_PERTURBATION
    blk = MeshBlock(p)
    dt = 0.5 * blk.new_dt()
    blk.close()
    ref = _block_two_steps(p, dt, reset_profile=p.cfg.precision == FP32_PERTURBATION)
    got = _noalloc_two_steps(p, dt)
    for call, ((ur, wr, er), (ug, wg, eg)) in enumerate(zip(ref, got)):
        assert er == 0 and eg == 0, (call, er, eg)
        assert np.array_equal(ur, ug), (call, float(np.abs(ur - ug).max()))
        # interior and ghost cells of w: ghosts are filled by the same kernel
        assert np.array_equal(wr, wg), (call, float(np.abs(wr - wg).max()))
    # the state did move
    assert not np.array_equal(got[1][0], p.u)


def test_noalloc_rejects_block_beyond_scratch():
    import torch
    lib = load()
    p = problems.moist3d(nx1=64, nx2=64, nx3=64)
    u = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.canoe_block_step_noalloc(ctypes.byref(p.cfg), u.data_ptr(), u.data_ptr(), None,
                                      1.0, None)
    assert rc == CANOE_ERR_ARG
    assert b"scratch" in lib.canoe_last_error()


def _small_moist():
    return problems.moist3d(nx1=24, nx2=16, nx3=12, x1max=3000.0, x2max=4000.0,
                            x3max=3000.0, noise=0.5)


def test_noalloc_rejects_what_block_create_rejects():
    """A configuration canoe_block_create refuses is refused here too, before
    any device work: an unknown reconstruction or Riemann solver, and PPM on
    a non-uniform x1 grid."""
    import torch
    lib = load()
    u = torch.zeros(1, dtype=torch.float64, device="cuda")

    def call(p):
        return lib.canoe_block_step_noalloc(ctypes.byref(p.cfg), u.data_ptr(), u.data_ptr(),
                                            None, 1.0, None)

    p = _small_moist()
    p.cfg.recon = 7
    assert call(p) == CANOE_ERR_ARG
    p = _small_moist()
    p.cfg.rsolver = 9
    assert call(p) == CANOE_ERR_ARG
    p = _small_moist()
    p.cfg.precision = 5
    assert call(p) == CANOE_ERR_ARG
    p = _small_moist()
    x1f = np.array(p.x1f, dtype=np.float64)
    x1f[1:-1] += 0.1 * np.diff(x1f)[:-1] * np.sin(np.arange(1, x1f.size - 1))
    p.x1f = np.ascontiguousarray(x1f)
    p.cfg.h_x1f = p.x1f.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert call(p) == CANOE_ERR_UNSUPPORTED
    assert b"uniform" in lib.canoe_last_error()


def test_noalloc_null_error_word_and_no_device_allocation():
    """With d_err = NULL the error bits stay in the library's scratch and the
    result is the same as with the caller's word; after one warm-up call, more
    calls leave the device's free memory unchanged (nothing is allocated)."""
    import torch
    lib = load()
    p = _small_moist()
    blk = MeshBlock(p)
    dt = 0.5 * blk.new_dt()
    blk.close()
    s = torch.cuda.current_stream()
    u0 = torch.from_numpy(np.ascontiguousarray(p.u)).cuda()

    def steps(use_err, n):
        u = u0.clone()
        w = torch.zeros_like(u)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        for _ in range(n):
            check(lib.canoe_block_step_noalloc(ctypes.byref(p.cfg), u.data_ptr(), w.data_ptr(),
                                               err.data_ptr() if use_err else None, float(dt),
                                               ctypes.c_void_p(s.cuda_stream)),
                  "canoe_block_step_noalloc")
        s.synchronize()
        return u, w

    u_ref, _ = steps(True, 2)
    # buffers for the measured calls exist before the free-memory reading
    u = u0.clone()
    w = torch.zeros_like(u)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        check(lib.canoe_block_step_noalloc(ctypes.byref(p.cfg), u.data_ptr(), w.data_ptr(),
                                           None, float(dt), ctypes.c_void_p(s.cuda_stream)),
              "canoe_block_step_noalloc")
    s.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)
    u_null, _ = steps(False, 2)
    assert torch.equal(u_null, u_ref)
