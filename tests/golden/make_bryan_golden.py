"""Generate the equivalent potential temperature of the moist rising-bubble
run (bryan.inp's configuration, canoe_b200.problems.bryan2d) computed by the
oracle on the host cores through the same main loop as the CUDA run
(canoe_b200.driver.evolve) and written by canoe_b200.output with the input's
output interval of 100 s:

    tests/golden/bryan2d_ppm.theta_e.00000-00300s.nc   records 0 .. 3 (t = 0,
        and the first cycles past 100, 200 and 300 s), the file test_bryan.py
        indexes as theta_e[3, 0, :, :]
    tests/golden/bryan2d_ppm.theta_e.01000s.nc         tlim = 1000 s

    python tests/golden/make_bryan_golden.py [--threads N]

About 15 k cycles of 200 x 400 cells: some 4 minutes on 8 cores.
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
    p = problems.bryan2d()
    ob = oracle.OracleBlock(p)
    t0 = time.time()
    tmp = tempfile.mkdtemp()
    o = output.NetcdfOutput(os.path.join(tmp, "bryan2d"), dt=p.meta["out_dt"], p0=p.meta["p0"],
                            variables=("theta_e",))
    t, cycles = driver.evolve(ob, p.meta["tlim"], [o])
    joined = os.path.join(a.out, "bryan2d_ppm.theta_e.00000-00300s.nc")
    output.join_records(o.written[:4], joined)
    last = os.path.join(a.out, "bryan2d_ppm.theta_e.01000s.nc")
    shutil.copy(o.written[-1], last)
    shutil.rmtree(tmp)
    print(joined, list(output.read_variable(joined, "time")))
    print(last, float(output.read_variable(last, "time")[0]))
    print(f"t = {t} s after {cycles} cycles, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
