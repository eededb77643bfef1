#!/usr/bin/env python3
"""Benchmark of the dynamical-core hot path: zone-cycles/s on B200.

A step is one full RK3 time step of the 3-D moist convection LES
(128 x 256 x 256 cells, 8 variables: dry air, H2O vapour / liquid / ice,
momentum, energy) with PPM reconstruction, the HLLC solver, the implicit
vertical block-tridiagonal correction and the saturation adjustment, i.e.
the task list of ImplicitHydroTasks.  A zone-cycle is one interior cell
advanced one step (canoe src/mesh_destroy.cpp:43-53).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) the ranks hold the N blocks of one periodic domain
cut along x2, each block the configuration's full 128 x 256 x 256 (weak
scaling): every RK stage exchanges the NGHOST ghost layers of the x2 block
sides between ranks by NCCL point-to-point transfers
(canoe_b200.distributed).  Rank 0 prints one JSON line.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-cycles/s on 1 B200: mixed+learned vs plain FP64 at stated L2 error"
UNIT = "zone-cycles/s"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples of this process's GPU (selected by
    UUID, so CUDA_VISIBLE_DEVICES remapping does not matter).  start() waits
    for the first sample; samples are time-stamped and those inside the
    timed region [mark_begin(), mark_end()] are reported (all samples under
    load when the region is shorter than the sampling period)."""

    def __init__(self, device=0, period_ms=100):
        self.device = device
        self.period_ms = period_ms
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def _gpu_id(self):
        import torch
        try:
            return "GPU-" + str(torch.cuda.get_device_properties(self.device).uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x.strip() for x in vis.split(",") if x.strip()]
            return ids[self.device] if self.device < len(ids) else str(self.device)

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self._gpu_id()}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.monotonic() + 10.0
            while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.05)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark_begin(self):
        self.t0 = time.monotonic()

    def mark_end(self):
        self.t1 = time.monotonic()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"],
                    "samples": 0}
        time.sleep(2.5 * self.period_ms * 1e-3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

        def parse(lines):
            sm, smax, reasons = [], None, set()
            for _, ln in lines:
                f = [x.strip() for x in ln.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = float(f[2])
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            return sm, smax, reasons

        window = "timed region"
        lo = (self.t0 or 0.0) - 0.5 * self.period_ms * 1e-3
        hi = (self.t1 or time.monotonic()) + 1.5 * self.period_ms * 1e-3
        sm, smax, reasons = parse([x for x in self.lines if lo <= x[0] <= hi])
        if not sm:
            window = "warm-up and timed region"
            sm, smax, reasons = parse(self.lines[1:])
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


def job_rates(ms_list, cells_per_rank, steps, dist=None, device="cuda"):
    """Max over ranks of each timed region (ms, CUDA events) and the
    whole-job zone-cycles/s: every rank advances its own replica of
    cells_per_rank cells (weak scaling, no data-path collective)."""
    import torch
    t = torch.tensor(ms_list, dtype=torch.float64, device=device)
    world = 1
    if dist is not None and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        world = dist.get_world_size()
    ms = [float(x) for x in t.tolist()]
    return ms, [world * cells_per_rank * steps / (m * 1e-3) for m in ms]


def make_problem(args, nx2=None, nx3=None, seed_offset=0):
    from canoe_b200 import problems
    return problems.moist3d(nx1=args.nx1, nx2=nx2 or args.nx2, nx3=nx3 or args.nx3,
                            x1max=16.0e3, x2max=64.0e3 * (nx2 or args.nx2) / 256,
                            x3max=64.0e3 * (nx3 or args.nx3) / 256,
                            implicit_flag=getattr(args, "implicit_flag", 1),
                            seed=20240601 + seed_offset)


def algorithmic_bytes(nv, ny, ncell):
    """bytes per launch of each kernel class: inputs read once, outputs written
    once, interior cells, 8-byte words."""
    return {
        # x1 pencil: read w, du (x2/x3 part), u, u1; write u (+ u1 at stage 0)
        "x1_pencil": (40 * nv + 8 * nv / 3.0) * ncell,
        "flux_x2": 16 * nv * ncell,            # read w; write du
        "flux_x3": 24 * nv * ncell,            # read w, du; write du
        "satadj": 8 * (nv + ny) * ncell,       # read u; write u[1..ny]
        "cons_to_prim": 16 * nv * ncell,       # read u; write w
    }


# kernel classes timed by canoe_block_step_profile
CLASSES = ["x1_pencil", "flux_x2", "flux_x3", "unused", "satadj", "cons_to_prim", "dt"]
LAUNCHES_PER_STEP = {"x1_pencil": 3, "flux_x2": 3, "flux_x3": 3, "unused": 0,
                     "satadj": 1, "cons_to_prim": 3, "dt": 1}


def cpu_baseline(args, reps=5, seconds_per_rep=2.0, patch=32):
    """The oracle (C++ restatement, OpenMP over all host threads) on a bounded
    sample of the workload: full 128-level columns on a patch x patch
    horizontal patch of the same configuration.  `reps` timed samples of at
    least `seconds_per_rep` each (whole steps) with every host thread, and
    `reps` single steps on one thread; each figure is the median of its
    samples."""
    from oracle import oracle
    nthreads = oracle.set_threads(os.cpu_count() or 1)
    p = make_problem(args, nx2=patch, nx3=patch)
    ob = oracle.OracleBlock(p)
    ncell = p.cfg.nx1 * p.cfg.nx2 * p.cfg.nx3
    ob.step(-1.0, 1)  # warm-up
    rates, steps = [], 0
    for _ in range(reps):
        t0 = time.perf_counter()
        n = 0
        while n < 1 or time.perf_counter() - t0 < seconds_per_rep:
            ob.step(-1.0, 1)
            n += 1
        rates.append(ncell * n / (time.perf_counter() - t0))
        steps += n
    oracle.set_threads(1)
    single = []
    for _ in range(reps):
        t0 = time.perf_counter()
        ob.step(-1.0, 1)
        single.append(ncell / (time.perf_counter() - t0))
    oracle.set_threads(nthreads)
    return {"value": float(np.median(rates)), "unit": UNIT, "cores": nthreads, "kind": "port",
            "single_thread": float(np.median(single)),
            "samples": [float(r) for r in rates],
            "sample": f"median of {reps} samples ({steps} steps in all) of a "
                      f"{p.cfg.nx1}x{patch}x{patch} patch of the same configuration "
                      f"({ncell} cells) on {nthreads} threads; single_thread: median of "
                      f"{reps} single steps on 1 thread"}


def c1_report(steps=2000, warmup=20, cpu_steps=200):
    """C1: the 2-D dry rising bubble, 150 x 100, PLM + LMARS, no implicit
    solve, FP64, every step with the device's CFL time step, stepped as a
    replayed CUDA graph for the configuration's 2000 steps; beside it the
    oracle on the host cores over `cpu_steps` steps of the same run."""
    import torch
    from canoe_b200 import MeshBlock, problems
    from canoe_b200._abi import check
    p = problems.bubble2d()
    cells = p.cfg.nx1 * p.cfg.nx2 * p.cfg.nx3
    stream = torch.cuda.Stream()
    blk = MeshBlock(p, graph=True)
    check(blk.lib.canoe_block_set_stream(blk.h, ctypes.c_void_p(stream.cuda_stream)))
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            blk.step()
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            blk.step()
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"config": "150 x 100 x 1, PLM + LMARS, FP64, no implicit solve, device CFL dt "
                     "(0.8 split over the 2 directions) every step, graph replay",
           "cells": cells, "steps": steps, "ms_per_step": ms / steps,
           "value": cells * steps / (ms * 1e-3), "unit": UNIT,
           "error_word": blk.error_word(),
           "finite": bool(np.isfinite(blk.conserved()).all())}
    blk.close()
    from oracle import oracle
    nthreads = oracle.set_threads(os.cpu_count() or 1)
    ob = oracle.OracleBlock(problems.bubble2d())
    ob.step(-1.0, 1)
    t0 = time.perf_counter()
    ob.step(-1.0, cpu_steps)
    el = time.perf_counter() - t0
    out["cpu_oracle"] = {"value": cells * cpu_steps / el, "cores": nthreads,
                         "sample": f"{cpu_steps} steps of the same run"}
    return out


def accuracy_report(args, net, nsteps):
    """The north star's accuracy statement on the headline configuration:
    the mixed + learned form and plain FP64 each advance C2 (full size) by
    `nsteps` steps of the same fixed dt (the CFL step of the initial state)
    from the same initial state; the relative L2 differences of potential
    temperature and total water, the drift of total mass and total water of
    each run, and the saturation adjustment's statistics over the run."""
    import torch
    from canoe_b200 import MeshBlock
    from canoe_b200 import thermo as T_
    from canoe_b200._abi import FP32_PERTURBATION, FP64
    p = make_problem(args)
    ny = p.ny
    th = p.cfg.thermo
    u0 = p.interior(p.u)
    mass0, water0 = float(u0[:1 + ny].sum()), float(u0[1:1 + ny].sum())
    del u0
    res, dt0 = {}, None
    for name, prec in (("fp64", FP64), ("mixed", FP32_PERTURBATION)):
        p.cfg.precision = prec
        b = MeshBlock(p, graph=True)
        if name == "mixed":
            b.set_mlp(net)
        dt0 = dt0 or b.new_dt()
        b.set_fixed_dt(dt0)
        b.satadj_stats()
        t0 = time.perf_counter()
        for _ in range(nsteps):
            b.step()
        b.synchronize()
        el = time.perf_counter() - t0
        s = b.satadj_stats()
        u = p.interior(b.conserved())
        w = p.interior(b.primitive())
        cfl_end = b.new_dt()
        vmax = float(np.abs(w[1 + ny:4 + ny]).max())
        q = w[1:1 + ny]
        T = w[4 + ny] / (w[0] * th.rd * T_.feps_of(th, q))
        kap = (th.gammad - 1.0) / th.gammad
        res[name] = {
            "theta": T * (1.0e5 / w[4 + ny]) ** kap, "water": u[1:1 + ny].sum(axis=0),
            "rec": {"wall_s": el, "error_word": b.error_word(),
                    "mass_drift": float(u[:1 + ny].sum()) / mass0 - 1.0,
                    "water_drift": float(u[1:1 + ny].sum()) / water0 - 1.0,
                    "max_speed_end": vmax, "cfl_dt_end": cfl_end,
                    "condensing_cells_end": int(((u[2:1 + ny] > 0).any(axis=0)).sum()),
                    "satadj_evaluations_per_cell": float(s[1]) / max(1, int(s[0])),
                    "satadj_fallback_rate": float(s[2]) / max(1, int(s[0])),
                    "satadj_not_converged": int(s[3])}}
        b.close()
        del u, w
        torch.cuda.empty_cache()

    def rl2(a, b):
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

    return {"steps": nsteps, "dt": dt0, "bar": 1e-4,
            "theta": rl2(res["mixed"]["theta"], res["fp64"]["theta"]),
            "total_water": rl2(res["mixed"]["water"], res["fp64"]["water"]),
            "fp64": res["fp64"]["rec"], "mixed": res["mixed"]["rec"],
            "note": "relative L2 of the mixed + learned run against the plain FP64 run "
                    "after the same steps; the FP64 GPU path matches the oracle to 1e-11 "
                    "per step (tests/test_gpu_fullsize_parity.py); total water changes "
                    "only through the implicit species correction of the reference "
                    "(forward_backward.hpp:101-124)"}


def c4_report(net, th, ncells=1 << 24, reps=3):
    """C4: the learned warm start on 16.8 M perturbed cells against the cold
    start: device time (one untimed call, then the mean of `reps` calls, each
    on a fresh copy of the same states), evaluations of the energy residual,
    fallbacks."""
    import torch
    from canoe_b200 import learned
    from canoe_b200._abi import SatOpts, check, load
    lib = load()
    u = learned.perturbed_states(th, ncells, seed=2024)
    src = torch.from_numpy(u).cuda()
    out = {"cells": ncells}
    for name, mode in (("cold", 0), ("learned", 2)):
        d = torch.empty_like(src)
        st = torch.zeros(4, dtype=torch.int64, device="cuda")
        o = SatOpts(1e-8, 30, mode)

        def call():
            if mode == 0:
                check(lib.canoe_saturation_adjust(ctypes.byref(th), ctypes.byref(o), d.data_ptr(),
                                                  ncells, None, None, None, st.data_ptr(), None))
            else:
                check(lib.canoe_saturation_adjust_learned(ctypes.byref(th), ctypes.byref(o),
                                                          net.h, d.data_ptr(), ncells, None,
                                                          None, st.data_ptr(), None, None))
        ms = 0.
        for r in range(reps + 1):
            d.copy_(src)
            st.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            call()
            e1.record()
            e1.synchronize()
            if r > 0:
                ms += e0.elapsed_time(e1) / reps
        s = st.cpu().numpy()
        out[name] = {"ms": ms, "evaluations_per_cell": float(s[1]) / s[0],
                     "fallback_rate": float(s[2]) / s[0], "not_converged": int(s[3])}
        del d
    # the network's inference alone over the same number of cells (seeded
    # normalised inputs): tcgen05 warpgroups against the FP32 CUDA cores
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    x = torch.randn(ncells, 4, device="cuda", dtype=torch.float32, generator=gen)
    y = torch.empty(ncells, device="cuda", dtype=torch.float32)
    inf = {}
    for name, tc in (("tcgen05", 1), ("fp32_cuda_cores", 0)):
        def fwd():
            check(lib.canoe_mlp_forward(net.h, x.data_ptr(), y.data_ptr(), ncells, tc, None))
        for _ in range(3):
            fwd()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fwd()
        e1.record()
        e1.synchronize()
        inf[name + "_ms"] = e0.elapsed_time(e1) / reps
        if tc:
            inf["finite"] = bool(torch.isfinite(y).all())
    inf["samples_per_s"] = ncells / (inf["tcgen05_ms"] * 1e-3)
    out["inference"] = inf
    del x, y
    out["note"] = ("same tolerance (1e-8 K + one polishing step) and the same answer; "
                   "the gated start uses the network where it predicts latent heating")
    return out


def c3_report(steps=10, warmup=3, nx1=64, nside=96, dt=60.0):
    """C3: the six-panel cubed-sphere shell (PPM + HLLC, implicit x1) stepped
    on device with the panel exchange, FP32 fluxes on the hydrostatic
    perturbation against plain FP64: zone-cycles/s of both, the L2 difference
    after the same steps, and the ghost exchange's bandwidth (algorithmic
    bytes: two source reads and one write of NV doubles per ghost cell)."""
    import torch
    from canoe_b200 import Shell, problems
    from canoe_b200._abi import check
    cells = 6 * nside * nside * nx1
    out = {"cells": cells, "config": f"6 x {nside}x{nside} x {nx1}, PPM + HLLC, implicit x1 "
           "partial 3x3", "dt": dt, "unit": UNIT}
    stream = torch.cuda.Stream()
    states = {}
    for name, prec in (("mixed", 1), ("fp64", 0)):
        p = problems.shell_c3(nx1=nx1, nside=nside)
        p.cfg.precision = prec
        sh = Shell(p)
        check(sh.lib.canoe_shell_set_stream(sh.h, ctypes.c_void_p(stream.cuda_stream)))
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                sh.step(dt)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                sh.step(dt)
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            rec = {"ms_per_step": ms / steps, "value": cells * steps / (ms * 1e-3)}
            if name == "fp64":
                # the ghost exchange alone, repeated (its inputs, the panels'
                # edge layers, 53 MB at full size, stay in L2)
                reps = 50
                e0.record(stream)
                for _ in range(reps):
                    check(sh.lib.canoe_shell_fill_ghosts(sh.h))
                e1.record(stream)
                e1.synchronize()
                us = e0.elapsed_time(e1) * 1e3 / reps
                ghosts = 6 * 4 * 3 * nside * nx1
                byts = 3 * 8 * 5 * ghosts
                out["ghost_exchange"] = {"us_per_call": us, "ghost_cells": ghosts,
                                         "algorithmic_bytes": byts,
                                         "gbs": byts / (us * 1e-6) / 1e9,
                                         "note": "repeated calls: source layers L2-resident"}
        states[name] = p.interior(sh.conserved())
        rec["finite"] = bool(np.isfinite(states[name]).all())
        rec["error_word"] = sh.error_word()
        out[name] = rec
        sh.close()
    a, b = states["mixed"], states["fp64"]
    out["l2_error_mixed_vs_fp64"] = {
        "density": float(np.linalg.norm(a[:, 0] - b[:, 0]) / np.linalg.norm(b[:, 0])),
        "momentum": float(np.linalg.norm(a[:, 1:4] - b[:, 1:4]) / np.linalg.norm(b[:, 1:4])),
        "energy": float(np.linalg.norm(a[:, 4] - b[:, 4]) / np.linalg.norm(b[:, 4])),
        "steps": warmup + steps}
    out["value"] = out["mixed"]["value"]
    out["ms_per_step"] = out["mixed"]["ms_per_step"]
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def full5x5_report(args, net, steps=5, warmup=2):
    """C2 with the full 5x5 implicit correction (implicit_flag 9, the
    FullCorrection of most of the reference's example inputs): mixed +
    learned against plain FP64, whole steps and the x1 pencil per launch."""
    import torch
    from canoe_b200 import MeshBlock
    from canoe_b200._abi import FP32_PERTURBATION, FP64, check, load
    lib = load()
    p = make_problem(args)
    p.cfg.implicit_flag = 9
    ncell = p.cfg.nx1 * p.cfg.nx2 * p.cfg.nx3
    stream = torch.cuda.Stream()
    out = {"config": f"{p.cfg.nx1}x{p.cfg.nx2}x{p.cfg.nx3}, PPM + HLLC, implicit x1 full 5x5",
           "unit": UNIT}
    states, dt0 = {}, None
    for name, prec in (("mixed", FP32_PERTURBATION), ("fp64", FP64)):
        p.cfg.precision = prec
        blk = MeshBlock(p, graph=True)
        check(lib.canoe_block_set_stream(blk.h, ctypes.c_void_p(stream.cuda_stream)))
        if name == "mixed":
            blk.set_mlp(net)
        dt0 = dt0 or blk.new_dt()
        blk.set_fixed_dt(dt0)
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                blk.step()
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                blk.step()
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            prof = (ctypes.c_float * 7)()
            check(lib.canoe_block_step_profile(blk.h, -1.0, prof, 7))
            stream.synchronize()
        rec = {"ms_per_step": ms / steps, "value": ncell * steps / (ms * 1e-3),
               "x1_pencil_ms_per_launch": prof[0] / 3, "error_word": blk.error_word()}
        states[name] = p.interior(blk.conserved())
        out[name] = rec
        blk.close()
    a, b = states["mixed"], states["fp64"]
    out["l2_error_mixed_vs_fp64"] = {
        "state": float(np.linalg.norm(a - b) / np.linalg.norm(b)),
        "steps": warmup + steps + 1}
    out["value"] = out["mixed"]["value"]
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def c5_report(net, steps=5, warmup=2):
    """C5: 48 uneven blocks of C2 physics stepped as one CUDA graph with
    autotuned threads per x1 pencil, mixed + learned and plain FP64, against
    the same blocks stepped one after another with default launches."""
    import torch
    from canoe_b200 import Batch, MeshBlock, problems
    ps = problems.batch_c5()
    cells = sum(p.cfg.nx1 * p.cfg.nx2 * p.cfg.nx3 for p in ps)
    out = {"blocks": len(ps), "cells": cells,
           "sizes": "nz logU[32,256], nh logU[16,128] square, seed 20240605"}

    def make(precision):
        blocks = []
        for p in ps:
            p.cfg.precision = 1 if precision == "mixed" else 0
            b = MeshBlock(p)
            if precision == "mixed":
                b.set_mlp(net)
            b.set_fixed_dt(b.new_dt())
            blocks.append(b)
        return blocks

    def timed(fn, sync):
        for _ in range(warmup):
            fn()
        sync()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        sync()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    for prec in ("mixed", "fp64"):
        blocks = make(prec)
        bt = Batch(blocks, graph=False)
        # one block after another on one stream, default launches
        def seq():
            for b in blocks:
                b.step()
                b.synchronize()
        ms_seq = timed(seq, lambda: None)
        choice = bt.autotune()
        bt.use_graph(True)
        ms_graph = timed(bt.step, bt.synchronize)
        errs = [b.error_word() for b in blocks]
        out[prec] = {"ms_per_step": ms_graph, "value": cells / (ms_graph * 1e-3),
                     "sequential_ms_per_step": ms_seq,
                     "sequential_value": cells / (ms_seq * 1e-3),
                     "threads_per_pencil": {str(t): int((choice == t).sum())
                                            for t in (64, 96, 128, 160, 192, 256)},
                     "cells_per_flux_run": {str(r): sum(1 for _, fr in bt.shapes() if fr == r)
                                            for r in (0, 8, 16, 32, 64)},
                     "error_words": int(np.bitwise_or.reduce(np.array(errs)))}
        bt.close()
        for b in blocks:
            b.close()
    out["unit"] = UNIT
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def run_reference(args, rank):
    if rank != 0:
        return
    cb = cpu_baseline(args, reps=max(3, min(args.steps, 5)))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(args),
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_partitioned(args, dist, rank, world):
    """N > 1: the ranks' blocks tile one periodic domain along x2 (block q on
    rank q, each the full configuration), stepped with the x2 ghost layers
    exchanged by NCCL every RK stage; both precisions, the mixed one with the
    learned warm start.  Timed on each rank with CUDA events on the stream
    that carries the kernels and the transfers, the max over ranks."""
    import torch
    from canoe_b200 import distributed, learned
    from canoe_b200._abi import BC_BLOCK, FP32_PERTURBATION, FP64
    net = learned.default_net()
    ncell = args.nx1 * args.nx2 * args.nx3
    neighbors = [{2: (q - 1) % world, 3: (q + 1) % world} for q in range(world)]
    order = [args.precision] + [k for k in ("fp64", "mixed") if k != args.precision]
    results, dt0, clocks = {}, None, None
    for name in order:
        p = make_problem(args, seed_offset=rank)
        p.cfg.precision = FP32_PERTURBATION if name == "mixed" else FP64
        p.cfg.bc[2] = p.cfg.bc[3] = BC_BLOCK
        dm = distributed.DistributedMesh({rank: p}, neighbors, list(range(world)),
                                         distributed.GpuBackend(), dist)
        if name == "mixed":
            dm.blocks[rank].set_mlp(net)
        dt0 = dt0 or dm.dt
        stream = torch.cuda.current_stream()
        sampler = ClockSampler(torch.cuda.current_device()) if name == args.precision else None
        if sampler:
            sampler.start()
        for _ in range(args.warmup):
            dm.step(dt0, update_dt=False)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.mark_begin()
        e0.record(stream)
        for _ in range(args.steps):
            dm.step(dt0, update_dt=False)
        e1.record(stream)
        e1.synchronize()
        if sampler:
            sampler.mark_end()
            clocks = sampler.stop()
        results[name] = (e0.elapsed_time(e1), dm.blocks[rank].error_word())
        dist.barrier()
        dm.close()
        torch.cuda.empty_cache()
    (ms, ms_o), (value, value_o) = job_rates([results[order[0]][0], results[order[1]][0]],
                                             ncell, args.steps, dist)
    dist.barrier()
    dist.destroy_process_group()
    if rank != 0:
        return
    cfg = config_dict(args)
    cfg["parallelism"] = (f"{world} GPUs, one 128x256x256 block each, periodic domain cut "
                          "along x2, NCCL halo exchange of 3 ghost layers every RK stage")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded C2 initial state per block)", "config": cfg,
            "gpu_launches": args.steps * 27,  # 15 kernels of the stages, 12 packs / unpacks
            "other_variant": {"variant": order[1], "value": value_o,
                              "ms_per_step": ms_o / args.steps},
            "roofline": None, "cpu_baseline": None, "e2e": None, "clocks": clocks,
            "error_word": int(results[order[0]][1])}
    print(json.dumps(line), flush=True)


def config_dict(args):
    return {"workload": f"C2 3-D moist convection LES {args.nx1}x{args.nx2}x{args.nx3}, "
                        "PPM + HLLC, implicit X1 "
                        + ("partial 3x3" if args.implicit_flag == 1 else "full 5x5")
                        + ", saturation adjustment each step",
            "cells": args.nx1 * args.nx2 * args.nx3, "nv": 8, "rk_stages": 3,
            "precision": {"fp64": "FP64", "mixed": "FP32 fluxes on the hydrostatic "
                          "perturbation, FP64 implicit / accumulation / saturation "
                          "adjustment"}[args.precision],
            "cfl": "0.8 split over the 2 horizontal directions (0.4 per direction)",
            "dt": "CFL step of the initial state, fixed",
            "l2_flush": "inputs larger than L2 (537 MB per state array)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx1", type=int, default=128)
    ap.add_argument("--nx2", type=int, default=256)
    ap.add_argument("--nx3", type=int, default=256)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="headline variant; the other one is timed alongside")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-c4", action="store_true")
    ap.add_argument("--no-c3", action="store_true")
    ap.add_argument("--no-c5", action="store_true")
    ap.add_argument("--implicit-flag", type=int, default=1, choices=[1, 9],
                    help="C2's implicit solve: 1 partial 3x3 (the headline), 9 full 5x5")
    ap.add_argument("--no-c1", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the mixed-vs-FP64 accuracy run on C2 (0: skip)")
    ap.add_argument("--no-5x5", action="store_true",
                    help="skip the full 5x5 implicit variant of C2")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the headline line; c1 / c3 / c4 / c5: only that report, as one "
                         "JSON line")
    ap.add_argument("--c4-cells", type=int, default=1 << 24,
                    help="cells of the C4 report (16.8 M by default)")
    args = ap.parse_args()
    if args.workload != "c2":
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        if args.workload == "c1":
            rep = c1_report()
        elif args.workload == "c3":
            rep = c3_report(steps=args.steps, warmup=args.warmup)
        elif args.workload == "c4":
            from canoe_b200 import learned, thermo
            rep = c4_report(learned.default_net(), thermo.earth_moist(), ncells=args.c4_cells)
        else:
            from canoe_b200 import learned
            rep = c5_report(learned.default_net(), steps=args.steps, warmup=args.warmup)
        print(json.dumps({"workload": args.workload, **rep}), flush=True)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if world > 1:
        run_partitioned(args, dist, rank, world)
        return

    from canoe_b200 import MeshBlock
    from canoe_b200._abi import FP32_PERTURBATION, FP64, check, load
    lib = load()
    p = make_problem(args)
    ncell = p.cfg.nx1 * p.cfg.nx2 * p.cfg.nx3
    nv, ny = p.nv, p.ny
    stream = torch.cuda.Stream()

    def make_block(prec):
        p.cfg.precision = prec
        b = MeshBlock(p, graph=True)
        check(lib.canoe_block_set_stream(b.h, ctypes.c_void_p(stream.cuda_stream)))
        return b

    from canoe_b200 import learned
    net = learned.default_net()
    blocks = {"fp64": make_block(FP64), "mixed": make_block(FP32_PERTURBATION)}
    # the headline: FP32 fluxes + learned warm start; plain FP64 alongside
    blocks["mixed"].set_mlp(net)
    # both variants step with the CFL time step of the initial state
    dt0 = blocks["fp64"].new_dt()
    for b in blocks.values():
        b.set_fixed_dt(dt0)
    order = [args.precision] + [k for k in blocks if k != args.precision]
    results, clocks = {}, None
    with torch.cuda.stream(stream):
        for name in order:
            blk = blocks[name]
            sampler = ClockSampler(torch.cuda.current_device()) if name == args.precision else None
            if sampler:
                sampler.start()
            for _ in range(args.warmup):
                blk.step()
            stream.synchronize()
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            if sampler:
                sampler.mark_begin()
            e0.record(stream)
            for _ in range(args.steps):
                blk.step()
            e1.record(stream)
            e1.synchronize()
            if sampler:
                sampler.mark_end()
            ms = e0.elapsed_time(e1)
            if sampler:
                clocks = sampler.stop()
            results[name] = {"ms": ms}
    # L2 error of the mixed run against the FP64 run: both took warmup+steps
    # steps of the same dt from the same state
    from canoe_b200 import thermo as T_
    wa, wb = p.interior(blocks["fp64"].primitive()), p.interior(blocks["mixed"].primitive())
    ua, ub = p.interior(blocks["fp64"].conserved()), p.interior(blocks["mixed"].conserved())

    def theta(w):
        q = w[1:1 + ny]
        T = w[4 + ny] / (w[0] * p.cfg.thermo.rd * T_.feps_of(p.cfg.thermo, q))
        kap = (p.cfg.thermo.gammad - 1.0) / p.cfg.thermo.gammad
        return T * (1.0e5 / w[4 + ny]) ** kap

    def rl2(a, b):
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

    l2 = {"theta": rl2(theta(wb), theta(wa)),
          "total_water": rl2(ub[1:1 + ny].sum(axis=0), ua[1:1 + ny].sum(axis=0)),
          "steps": args.warmup + args.steps}
    sat = {}
    for name, b in blocks.items():
        s = b.satadj_stats()
        sat[name] = {"evaluations_per_cell": float(s[1]) / max(1, int(s[0])),
                     "fallback_rate": float(s[2]) / max(1, int(s[0])),
                     "not_converged": int(s[3])}
    del wa, wb, ua, ub
    # per-kernel-class timing pass of the headline variant
    blk = blocks[args.precision]
    prof = (ctypes.c_float * 7)()
    nprof = max(2, min(args.steps, 5))
    with torch.cuda.stream(stream):
        for _ in range(nprof):
            check(lib.canoe_block_step_profile(blk.h, -1.0, prof, 7))
        stream.synchronize()
    launches = args.steps * sum(LAUNCHES_PER_STEP.values())
    err = blk.error_word()
    (ms, ms_other), (value, value_other) = job_rates(
        [results[args.precision]["ms"], results[order[1]]["ms"]], ncell, args.steps, dist)
    ms_step = ms / args.steps
    other = {"variant": order[1], "value": value_other, "ms_per_step": ms_other / args.steps}

    # roofline of the dominant kernel class
    hbm, peak_kind = peaks()
    abytes = algorithmic_bytes(nv, ny, ncell)
    per_class = {}
    for c, name in enumerate(CLASSES):
        nl = LAUNCHES_PER_STEP[name]
        if nl == 0:
            continue
        tot = prof[c] / nprof
        per_class[name] = {"ms_per_step": tot, "ms_per_launch": tot / nl}
        if name in abytes and tot > 0:
            per_class[name]["gbs"] = abytes[name] / (tot / nl * 1e-3) / 1e9
    dom = max((n for n in per_class if n in abytes), key=lambda n: per_class[n]["ms_per_step"])
    ach = per_class[dom]["gbs"]
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf)).get(args.precision, {}).get(dom)
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "traffic": traffic, "peak_kind": peak_kind,
                "algorithmic_bytes_per_launch": abytes[dom], "per_kernel": per_class}
    p.cfg.precision = blk.problem.cfg.precision

    # end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        hu = torch.empty(p.u.shape, dtype=torch.float64).pin_memory()
        hu.numpy()[...] = p.u
        ho = torch.empty(p.u.shape, dtype=torch.float64).pin_memory()
        blk = blocks[args.precision]
        torch.cuda.synchronize()
        k = args.steps
        t0 = time.perf_counter()
        check(lib.canoe_block_set_conserved(blk.h, ctypes.c_void_p(hu.data_ptr())))
        dtv = ctypes.c_double()
        for _ in range(k):
            check(lib.canoe_block_step(blk.h, -1.0))
            check(lib.canoe_block_new_dt(blk.h, ctypes.byref(dtv)))
        check(lib.canoe_block_get_conserved(blk.h, ctypes.c_void_p(ho.data_ptr())))
        el = time.perf_counter() - t0
        nbytes = hu.numel() * 8
        e2e = {"value": world * ncell * k / el, "unit": UNIT,
               "h2d_bytes_per_step": nbytes / k, "d2h_bytes_per_step": nbytes / k + 8,
               "note": "state uploaded once and downloaded once per K-step run "
                       "(bytes amortised per step); dt read back every step"}
        # K = 1 per call: the whole state up, one step, the whole state down,
        # as a host that keeps its own arrays would call it at every step
        k1 = max(3, min(k, 10))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k1):
            check(lib.canoe_block_set_conserved(blk.h, ctypes.c_void_p(hu.data_ptr())))
            check(lib.canoe_block_step(blk.h, -1.0))
            check(lib.canoe_block_get_conserved(blk.h, ctypes.c_void_p(ho.data_ptr())))
        el1 = time.perf_counter() - t0
        e2e["per_call"] = {"value": world * ncell * k1 / el1, "unit": UNIT, "calls": k1,
                           "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                           "note": "every call uploads the state from pinned memory, steps "
                                   "once and downloads the state"}

    # the single-GPU reports run at N = 1 only (with N > 1 the other ranks
    # would wait on rank 0 at the closing barrier)
    solo = rank == 0 and world == 1
    cb = None
    if solo and not args.no_cpu_baseline:
        cb = cpu_baseline(args)
    c4 = None
    c3 = None
    if solo and not args.no_c3:
        c3 = c3_report()
    c1 = None
    if solo and not args.no_c1:
        c1 = c1_report()
    acc = None
    if solo and args.accuracy_steps > 0:
        acc = accuracy_report(args, net, args.accuracy_steps)
    c5 = None
    if solo and not args.no_c5:
        c5 = c5_report(net)
    f5 = None
    if solo and not args.no_5x5:
        f5 = full5x5_report(args, net)
    fma = None
    if solo:
        # non-tensor FMA peaks of this GPU (outside every timed region): the
        # denominator for the x1 pencil's FP64 arithmetic in profiles/
        p64, p32 = ctypes.c_double(0.), ctypes.c_double(0.)
        check(lib.canoe_measure_fma_peak(0, ctypes.byref(p64)))
        check(lib.canoe_measure_fma_peak(1, ctypes.byref(p32)))
        fma = {"fp64_tflops": p64.value, "fp32_tflops": p32.value,
               "how": "8 independent FMA chains per thread, 8 CTAs x 256 threads per SM, "
                      "CUDA events after a warm-up launch"}
    if solo and not args.no_c4:
        c4 = c4_report(net, p.cfg.thermo)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded C2 initial state)",
            "config": config_dict(args), "gpu_launches": launches,
            "other_variant": other, "speedup_mixed_vs_fp64":
                (value / other["value"]) if args.precision == "mixed" else other["value"] / value,
            "l2_error_mixed_vs_fp64": l2, "saturation_adjustment": sat,
            "accuracy_mixed_vs_fp64": acc,
            "c1_dry_bubble": c1,
            "c4_learned_warm_start": c4,
            "c3_cubed_sphere_shell": c3,
            "c5_batched_blocks": c5,
            "c2_full5x5": f5,
            "fma_peaks": fma,
            "roofline": roofline, "cpu_baseline": cb, "e2e": e2e, "clocks": clocks,
            "error_word": err}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
