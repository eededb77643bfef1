"""The committed golden fixtures (tests/golden/golden.npz, made by
tests/golden/make_golden.py from the oracle) against the oracle rerun now:
a regression pin of the oracle and of the seeded problem generators."""
import os
import sys

import numpy as np
import pytest

from canoe_b200 import thermo
from conftest import rel_l2

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

GOLD = os.path.join(HERE, "golden", "golden.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_generators_reproduce_inputs(gold):
    for name, make in (("c1", mg.small_c1), ("c2", mg.small_c2)):
        p = make()
        assert np.array_equal(p.interior(p.u), gold[f"{name}_gen"]), name
        assert np.array_equal(mg.perturb(p), gold[f"{name}_u0"]), name
    p = mg.small_c3()
    assert np.array_equal(p.interior(p.u), gold["c3_u0"])


def test_riemann(gold, oracle_mod):
    th = thermo.earth_moist()
    wl, wr = mg.random_faces(th, 256, seed=101)
    assert np.array_equal(wl, gold["riemann_wl"]) and np.array_equal(wr, gold["riemann_wr"])
    for name, rs in (("lmars", 0), ("hllc", 1)):
        for d in range(3):
            got = oracle_mod.riemann(rs, th, 1 + th.ny + d, wl, wr)
            assert rel_l2(got, gold[f"riemann_{name}_x{d + 1}"]) < 1e-14


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_block_step(gold, oracle_mod, name):
    oracle_mod.set_threads(1)
    p = mg.with_interior({"c1": mg.small_c1, "c2": mg.small_c2}[name](), gold[f"{name}_u0"])
    ob = oracle_mod.OracleBlock(p)
    ob.step(float(gold[f"{name}_dt"]))
    assert rel_l2(p.interior(ob.conserved()), gold[f"{name}_u1"]) < 1e-13


def test_satadj(gold, oracle_mod):
    th = thermo.earth_moist()
    u = gold["satadj_u0"].copy()
    T, _, _ = oracle_mod.satadj(th, u)
    assert rel_l2(u, gold["satadj_u1"]) < 1e-14
    assert rel_l2(T, gold["satadj_T"]) < 1e-14


def test_shell(gold, oracle_mod):
    p = mg.small_c3()
    s = oracle_mod.OracleShell(p)
    s.set_conserved(p.u, fill=False)
    s.fill_ghosts()
    g = s.conserved()
    ng, n = 3, p.cfg.nside
    a, lo, hi = slice(ng, ng + n), slice(0, ng), slice(ng + n, 2 * ng + n)
    i = slice(ng, ng + p.cfg.nx1)
    for key, got in (("x2lo", g[:, :, a, lo, i]), ("x2hi", g[:, :, a, hi, i]),
                     ("x3lo", g[:, :, lo, a, i]), ("x3hi", g[:, :, hi, a, i])):
        assert rel_l2(got, gold[f"exo3_ghost_{key}"]) < 1e-14, key
    s = oracle_mod.OracleShell(p)
    s.step(float(gold["c3_dt"]))
    assert rel_l2(p.interior(s.conserved()), gold["c3_u1"]) < 1e-13
