"""The CUDA path against the committed golden fixtures (oracle outputs on
seeded inputs, tests/golden/make_golden.py), at the parity bars of the
oracle tests; nothing here runs the oracle."""
import ctypes
import os
import sys

import numpy as np
import pytest

from canoe_b200 import MeshBlock, Shell, learned, thermo
from canoe_b200._abi import check, load
from conftest import max_var_rel_l2, rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(HERE, "golden", "golden.npz"))


def test_riemann(gold):
    import torch
    th = thermo.earth_moist()
    lib = load()
    dl = torch.from_numpy(gold["riemann_wl"]).cuda()
    dr = torch.from_numpy(gold["riemann_wr"]).cuda()
    n = dl.shape[1]
    for name, fn in (("lmars", lib.canoe_riemann_lmars), ("hllc", lib.canoe_riemann_hllc)):
        for d in range(3):
            df = torch.zeros_like(dl)
            torch.cuda.synchronize()
            check(fn(ctypes.byref(th), 1 + th.ny + d, dl.data_ptr(), dr.data_ptr(),
                     df.data_ptr(), n, None))
            torch.cuda.synchronize()
            ref = gold[f"riemann_{name}_x{d + 1}"]
            scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
            assert np.max(np.abs(df.cpu().numpy() - ref) / scale) < 1e-13, (name, d)


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_block_step(gold, name):
    p = mg.with_interior({"c1": mg.small_c1, "c2": mg.small_c2}[name](), gold[f"{name}_u0"])
    b = MeshBlock(p)
    b.step(float(gold[f"{name}_dt"]))
    got = p.interior(b.conserved())
    assert rel_l2(got, gold[f"{name}_u1"]) < 1e-11
    assert max_var_rel_l2(got, gold[f"{name}_u1"]) < 5e-11


def test_satadj(gold):
    th = thermo.earth_moist()
    u1, T, _, _, _ = learned.satadj_gpu(th, gold["satadj_u0"])
    assert rel_l2(u1, gold["satadj_u1"]) < 1e-12
    assert rel_l2(T, gold["satadj_T"]) < 1e-12


def test_shell(gold):
    p = mg.small_c3()
    sh = Shell(p, fill=False)
    sh.set_conserved(p.u, fill=False)
    sh.fill_ghosts()
    g = sh.conserved()
    ng, n = 3, p.cfg.nside
    a, lo, hi = slice(ng, ng + n), slice(0, ng), slice(ng + n, 2 * ng + n)
    i = slice(ng, ng + p.cfg.nx1)
    for key, got in (("x2lo", g[:, :, a, lo, i]), ("x2hi", g[:, :, a, hi, i]),
                     ("x3lo", g[:, :, lo, a, i]), ("x3hi", g[:, :, hi, a, i])):
        assert rel_l2(got, gold[f"exo3_ghost_{key}"]) < 1e-12, key
    sh = Shell(p)
    sh.step(float(gold["c3_dt"]))
    got = p.interior(sh.conserved())
    for v in range(5):
        assert rel_l2(got[:, v], gold["c3_u1"][:, v]) < 5e-11, v
