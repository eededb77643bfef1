"""The oracle's x2 / x3 implicit solves, pinned to its x1 solve (CPU only).

SolveImplicit3D (canoe src/snap/implicit/solve_implicit_3d.cpp:19-142) runs
the same PartialCorrection / FullCorrection along x3 and x2 on a transposed
du, with the velocity in the direction's frame.  Without gravity and with
equal spacings, an x2 (x3) solve of a state must therefore equal the x1
solve of the state with the x1 and x2 (x3) axes and velocities exchanged.
The x1 solve is the one pinned by the golden vectors and the GPU parity.
"""
import numpy as np
import pytest

from canoe_b200 import problems, thermo
from canoe_b200._abi import BC_PERIODIC, BC_REFLECT
from oracle.oracle import OracleBlock

NG = 3


def _box(n, bc):
    p = problems.periodic_x1(nx1=n, nx2=n, nx3=n, x1max=100.0 * n, x2max=100.0 * n,
                             x3max=100.0 * n, moist=False)
    for q in range(6):
        p.cfg.bc[q] = bc
    return p


def _swap(a, d):
    """exchange axis x1 with x(d+1) of a (NV, nc3, nc2, nc1) array and the
    matching velocity slots"""
    ax = {1: 2, 2: 1}[d]
    b = np.swapaxes(a, ax, 3).copy()
    b[[1, 1 + d]] = b[[1 + d, 1]]
    return b


@pytest.mark.parametrize("bc", [BC_PERIODIC, BC_REFLECT])
@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("d", [1, 2])
def test_line_solve_equals_transposed_x1(bc, full, d):
    n = 8
    p = _box(n, bc)
    rng = np.random.Generator(np.random.PCG64(5 + d))
    du = np.zeros(p.u.shape)
    p.interior(du)[...] = 1e-3 * rng.standard_normal(p.interior(du).shape) * \
        np.abs(p.interior(p.u)).mean(axis=(1, 2, 3))[:, None, None, None]
    dt = 3.0
    p.cfg.implicit_flag = (1 << d) | (8 if full else 0)
    got = OracleBlock(p).solve_implicit(du, dt)
    q = _box(n, bc)
    q.u = _swap(p.u, d)
    q.cfg.implicit_flag = 1 | (8 if full else 0)
    ref = _swap(OracleBlock(q).solve_implicit(_swap(du, d), dt), d)
    # IDN, the normal momentum and IEN are written back; the rest of du stays
    for s in (0, 1 + d, 4):
        a, b = p.interior(got)[s], p.interior(ref)[s]
        # the FP64 bar: the 5x5 pivots see the transverse unknowns permuted
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max(), s
    for s in {1, 2, 3} - {1 + d}:
        assert np.array_equal(p.interior(got)[s], p.interior(du)[s])
    # the solve did act
    assert not np.allclose(p.interior(got)[1 + d], p.interior(du)[1 + d])


def test_line_solves_run_x3_x2_x1_in_order():
    """all three bits: X3, then X2, then X1 on the running du"""
    p = _box(8, BC_PERIODIC)
    rng = np.random.Generator(np.random.PCG64(9))
    du = np.zeros(p.u.shape)
    p.interior(du)[...] = 1e-3 * rng.standard_normal(p.interior(du).shape) * \
        np.abs(p.interior(p.u)).mean(axis=(1, 2, 3))[:, None, None, None]
    step = {}
    for f in (4, 2, 1):
        p.cfg.implicit_flag = f
        step[f] = OracleBlock(p)
    d3 = step[4].solve_implicit(du, 2.0)
    d2 = step[2].solve_implicit(d3, 2.0)
    d1 = step[1].solve_implicit(d2, 2.0)
    p.cfg.implicit_flag = 7
    allb = OracleBlock(p).solve_implicit(du, 2.0)
    assert np.array_equal(allb, d1)


def test_moist_line_solves_are_refused():
    p = problems.periodic_x1(nx1=8, nx2=8, nx3=4, moist=True, implicit_flag=2)
    with pytest.raises(AssertionError, match="dry Cartesian"):
        OracleBlock(p).solve_implicit(np.zeros(p.u.shape), 1.0)
