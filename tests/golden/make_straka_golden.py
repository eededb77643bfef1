"""Generate the potential temperature of the dense sinking bubble run
(straka.inp's configuration, canoe_b200.problems.straka2d, with the
example's dissipation source of diffusivity 75 m^2/s) computed by the oracle
on the host cores through the same main loop as the CUDA run
(canoe_b200.driver.evolve) and written by canoe_b200.output with the
input's output interval of 300 s:

    tests/golden/straka2d_ppm.theta.00300s.nc   the first cycle past 300 s
    tests/golden/straka2d_ppm.theta.00900s.nc   tlim = 900 s

    python tests/golden/make_straka_golden.py [--threads N]

About 7.5 k cycles of 64 x 256 cells: some 20 seconds on 8 cores.
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
    p = problems.straka2d()
    ob = oracle.OracleBlock(p)
    ob.set_diffusion(p.meta["K"], p.meta["p0"])
    t0 = time.time()
    tmp = tempfile.mkdtemp()
    o = output.NetcdfOutput(os.path.join(tmp, "straka2d"), dt=p.meta["out_dt"], p0=p.meta["p0"],
                            variables=("uov",), only=("theta",))
    t, cycles = driver.evolve(ob, p.meta["tlim"], [o])
    for number, name in ((1, "00300s"), (len(o.written) - 1, "00900s")):
        dst = os.path.join(a.out, f"straka2d_ppm.theta.{name}.nc")
        shutil.copy(o.written[number], dst)
        print(dst, float(output.read_variable(dst, "time")[0]))
    shutil.rmtree(tmp)
    print(f"t = {t} s after {cycles} cycles, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
