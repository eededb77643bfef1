"""The oracle's periodic-x1 implicit solve (CPU only).

The restatement of PeriodicForwardSweep / PeriodicBackwardSubstitution
(canoe src/snap/implicit/periodic_forward_backward.hpp:15-234) is pinned
against a dense solve of the cyclic block-tridiagonal system it is meant to
solve, with the reference's corner convention: row is couples to ie through
b[is], row ie to is through c[is-1].  On a whole block the periodic step is
checked for what periodicity implies: a state rolled along x1 steps to the
rolled result.
"""
import numpy as np
import pytest

from canoe_b200 import problems
from oracle.oracle import OracleBlock, periodic_block_solve


def _dense(a, b, c, rhs):
    n, N = a.shape[0] - 1, a.shape[1]
    M = np.zeros((n * N, n * N))
    for i in range(1, n + 1):
        r = slice((i - 1) * N, i * N)
        M[r, r] = a[i]
        left = i - 1 if i > 1 else n       # b[1] is the upper corner
        right = i + 1 if i < n else 1      # c[0] is the lower corner
        M[r, (left - 1) * N:left * N] += b[i]
        M[r, (right - 1) * N:right * N] += c[i] if i < n else c[0]
    return np.linalg.solve(M, rhs[1:].reshape(-1)).reshape(n, N)


@pytest.mark.parametrize("N", [3, 5])
@pytest.mark.parametrize("n", [3, 4, 7, 16, 33])
def test_periodic_block_solve_matches_dense(N, n):
    rng = np.random.Generator(np.random.PCG64(1000 * N + n))
    a = rng.uniform(-1, 1, (n + 1, N, N)) + 4.0 * N * np.eye(N)
    b = rng.uniform(-1, 1, (n + 1, N, N))
    c = rng.uniform(-1, 1, (n + 1, N, N))
    rhs = rng.uniform(-1, 1, (n + 1, N))
    x = periodic_block_solve(a, b, c, rhs)
    ref = _dense(a, b, c, rhs)
    err = np.abs(x[1:] - ref).max() / np.abs(ref).max()
    assert err < 1e-13, err


def test_periodic_block_solve_rejects_short_columns():
    z = np.zeros((3, 3, 3))
    with pytest.raises(ValueError):
        periodic_block_solve(z + np.eye(3), z, z, np.zeros((3, 3)))


def _interior_step(p, dt):
    ob = OracleBlock(p)
    ob.step(dt)
    return p.interior(ob.conserved())


@pytest.mark.parametrize("flag,moist", [(1, False), (9, False), (1, True), (9, True)])
def test_periodic_step_commutes_with_roll(flag, moist):
    p = problems.periodic_x1(nx1=16, nx2=4, nx3=2, x1max=1600.0, moist=moist,
                             implicit_flag=flag)
    dt = 0.5 * OracleBlock(p).new_dt()
    base = _interior_step(p, dt)
    q = problems.periodic_x1(nx1=16, nx2=4, nx3=2, x1max=1600.0, moist=moist,
                             implicit_flag=flag)
    ng = 3
    q.u[..., ng:ng + 16] = np.roll(p.u[..., ng:ng + 16], 5, axis=-1)
    rolled = _interior_step(q, dt)
    for n in range(p.nv):
        ref = np.roll(base[n], 5, axis=-1)
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(rolled[n] - ref).max() / scale < 1e-12, n
    # the implicit correction did act: the explicit step differs
    p.cfg.implicit_flag = 0
    assert not np.allclose(_interior_step(p, dt), base, rtol=1e-9, atol=0)
