"""Generate the golden fixtures of tests/golden from the CPU oracle.

    python tests/golden/make_golden.py

The reference ships no outputs for this path (its unit tests are disabled
and its regression outputs are Git-LFS pointers), so these fixtures are the
oracle's outputs on seeded inputs: they pin the oracle against regressions
and let the device tests compare with fixed data.  Interior cells only
(ghosts are zero on input); every seed is recorded in the file.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from canoe_b200 import problems, thermo  # noqa: E402
from oracle import oracle  # noqa: E402


def random_faces(th, n, seed):
    """left / right primitive face states (NV, n) of moist air"""
    rng = np.random.Generator(np.random.PCG64(seed))
    ny = th.ny
    out = []
    for _ in range(2):
        w = np.zeros((5 + ny, n))
        w[0] = rng.uniform(0.2, 1.5, n)
        for s in range(1, ny + 1):
            w[s] = rng.uniform(0.0, 0.02, n)
        for s in range(1 + ny, 4 + ny):
            w[s] = rng.uniform(-60.0, 60.0, n)
        w[4 + ny] = rng.uniform(2.0e4, 1.2e5, n)
        out.append(w)
    return out


def perturb(p, seed=7, dv=0.5, drho=0.01, dp=0.002):
    """seeded perturbation of a problem's interior primitive state
    (velocities, density, pressure) so every flux component is exercised;
    returns the conserved interior state"""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = p.interior(p.w).copy()
    ny = p.ny
    w[0] *= 1.0 + drho * rng.uniform(-1, 1, w[0].shape)
    for n in range(1 + ny, 4 + ny):
        w[n] += dv * rng.uniform(-1, 1, w[n].shape)
    w[4 + ny] *= 1.0 + dp * rng.uniform(-1, 1, w[0].shape)
    if p.cfg.nx3 == 1:
        w[3 + ny] = 0.0
    return thermo.prim_to_cons(p.cfg.thermo, w)


def with_interior(p, u_int):
    """the problem with its interior conserved state replaced"""
    u = np.zeros_like(p.u)
    p.interior(u)[...] = u_int
    p.u = u
    return p


def small_c1():
    return problems.bubble2d(nx1=40, nx2=24, x1max=400.0, x2max=240.0)


def small_c2():
    return problems.moist3d(nx1=16, nx2=8, nx3=8, x1max=2000.0, x2max=2000.0, x3max=2000.0,
                            noise=0.5)


def small_c3():
    return problems.shell_c3(nx1=8, nside=8)


def main():
    oracle.set_threads(1)
    out = {}
    # Riemann solvers on random faces, every direction
    th = thermo.earth_moist()
    wl, wr = random_faces(th, 256, seed=101)
    for name, rs in (("lmars", 0), ("hllc", 1)):
        for d in range(3):
            out[f"riemann_{name}_x{d + 1}"] = oracle.riemann(rs, th, 1 + th.ny + d, wl, wr)
    out["riemann_wl"], out["riemann_wr"] = wl, wr
    # one step of C1 and of C2 at a fixed dt
    for name, make, dt in (("c1", small_c1, 0.2), ("c2", small_c2, 0.5)):
        p = make()
        out[f"{name}_gen"] = p.interior(p.u)
        p = with_interior(p, perturb(p))
        ob = oracle.OracleBlock(p)
        ob.step(dt)
        out[f"{name}_u0"] = p.interior(p.u)
        out[f"{name}_u1"] = p.interior(ob.conserved())
        out[f"{name}_dt"] = np.array(dt)
    # saturation adjustment of perturbed moist cells
    from canoe_b200 import learned
    u = learned.perturbed_states(th, 512, seed=202)
    out["satadj_u0"] = u.copy()
    T, it, _ = oracle.satadj(th, u)
    out["satadj_u1"], out["satadj_T"] = u, T
    # cubed-sphere ghost exchange and one shell step
    p = small_c3()
    s = oracle.OracleShell(p)
    s.set_conserved(p.u, fill=False)
    s.fill_ghosts()
    g = s.conserved()
    ng, n = 3, p.cfg.nside
    a, lo, hi = slice(ng, ng + n), slice(0, ng), slice(ng + n, 2 * ng + n)
    i = slice(ng, ng + p.cfg.nx1)
    out["exo3_ghost_x2lo"] = g[:, :, a, lo, i]
    out["exo3_ghost_x2hi"] = g[:, :, a, hi, i]
    out["exo3_ghost_x3lo"] = g[:, :, lo, a, i]
    out["exo3_ghost_x3hi"] = g[:, :, hi, a, i]
    s = oracle.OracleShell(p)
    s.step(5.0)
    out["c3_u0"] = p.interior(p.u)
    out["c3_u1"] = p.interior(s.conserved())
    out["c3_dt"] = np.array(5.0)
    out["seeds"] = np.array([101, 202, 20240601, 20240607])
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
