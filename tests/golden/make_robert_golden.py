"""Generate the potential temperature of the rising-bubble regression run
(robert2d.inp's configuration, canoe_b200.problems.robert2d) computed by the
oracle on the host cores through the same main loop as the CUDA run
(canoe_b200.driver.evolve) and written by canoe_b200.output with the
input's output interval of 180 s:

    tests/golden/robert2d_ppm.theta.00180s.nc   the first cycle past 180 s
    tests/golden/robert2d_ppm.theta.01080s.nc   tlim = 1080 s

    python tests/golden/make_robert_golden.py [--threads N]

About 170 k cycles of 300 x 200 cells: some 40 minutes on 8 cores.
"""
import argparse
import os
import shutil
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    from canoe_b200 import driver, output, problems
    from oracle import oracle
    oracle.set_threads(a.threads)
    p = problems.robert2d()
    ob = oracle.OracleBlock(p)
    t0 = time.time()
    tmp = tempfile.mkdtemp()
    o = output.NetcdfOutput(os.path.join(tmp, "robert2d"), dt=p.meta["out_dt"], p0=p.meta["p0"],
                            variables=("uov",), only=("theta",))
    t, cycles = driver.evolve(ob, p.meta["tlim"], [o])
    for number, name in ((1, "00180s"), (len(o.written) - 1, "01080s")):
        dst = os.path.join(a.out, f"robert2d_ppm.theta.{name}.nc")
        shutil.copy(o.written[number], dst)
        print(dst, float(output.read_variable(dst, "time")[0]))
    shutil.rmtree(tmp)
    print(f"t = {t} s after {cycles} cycles, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
