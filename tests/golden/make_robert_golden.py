"""Generate tests/golden/robert2d_ppm.theta.01080s.nc: the potential
temperature of the rising-bubble regression run (robert2d.inp's
configuration, canoe_b200.problems.robert2d) at tlim = 1080 s, computed by
the oracle on the host cores through the same main loop as the CUDA run
(canoe_b200.driver.evolve) and written by canoe_b200.output.

    python tests/golden/make_robert_golden.py [--threads N]

About 170 k cycles of 300 x 200 cells: some 25 minutes on 8 cores.
"""
import argparse
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

OUT = os.path.join(HERE, "robert2d_ppm.theta.01080s.nc")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=OUT)
    a = ap.parse_args()
    from canoe_b200 import driver, output, problems
    from oracle import oracle
    oracle.set_threads(a.threads)
    p = problems.robert2d()
    ob = oracle.OracleBlock(p)
    t0 = time.time()
    t, cycles = driver.evolve(ob, p.meta["tlim"])
    w = ob.primitive()
    fields = output.cell_fields(p.cfg, w, ("uov",), p.meta["p0"])
    output.write_file(a.out, output.coordinates(p.cfg, p.x1f), {"theta": fields["theta"]}, t)
    print(f"{a.out}: t = {t} s after {cycles} cycles, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
