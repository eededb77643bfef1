"""Train the saturation-adjustment warm-start network on the GPU and save it.

    python -m canoe_b200.train_warm_start [out.npz] [--pairs N] [--epochs E]

Training pairs: 16 M (the default --pairs) perturbed states of the moist
LES column (temperature +-10 K, total water x (1 +- 0.2)), labelled by the
plain cold-start Newton solve of the CUDA library; the fit runs on the
library's own FP32 forward / backward and Adam kernels (30 epochs of 16 M
pairs take about 25 s on one B200; held-out RMS 0.009 K).  The default output is the network the benchmark
and the block step use, canoe_b200/data/warm_start_c2.npz.
"""
import argparse
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT = os.path.join(HERE, "data", "warm_start_c2.npz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out", nargs="?", default=DEFAULT)
    ap.add_argument("--pairs", type=int, default=1 << 24)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args()
    import numpy as np
    from canoe_b200 import learned, thermo
    th = thermo.earth_moist()
    t0 = time.time()
    net = learned.train_warm_start(th, n=a.pairs, seed=a.seed, epochs=a.epochs, batch=a.batch,
                                   log=print)
    x, T = learned.training_pairs(th, 1 << 18, seed=a.seed + 1000)
    rms = float(np.sqrt(np.mean((learned.predict(net, th, x) - T) ** 2)))
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    net.save(a.out)
    print(f"saved {a.out}: held-out RMS {rms:.4f} K, {time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
