"""Benchmark: converged sweep points/s of the sweep-lane Newton path on B200.

    python bench.py --gpus N --steps K --warmup W [--impl reference]

A step is one pass of the hot path over one batch of lanes: every lane (one
sweep point) runs its whole Newton solve in the fused CUDA kernel. `value`
is device-timed (CUDA events on the library's stream, inputs resident in
HBM, L2 flushed between steps); `e2e` is the same metric through the public
C ABI with host buffers (start points in, solutions and statuses out,
copies inside the timed call). Under torchrun each rank solves its own batch
(independent points: no collective on the data path, weak scaling); the
times are the max over ranks.

--impl reference times the reference's CPU algorithm on this host's cores
(the C restatement under oracle/, since the Zig reference cannot be built
here), one point per worker thread as the reference's sweep pool runs them.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged sweep points/s on 1 B200, learned+mixed vs plain FP64 at 1e-9 rel"
UNIT = "points/s"


def workload(seed=1):
    from espice_b200 import decks
    fr, slots, values = decks.grid_diodes(seed=seed, points=256)
    cfg = {"workload": "grid_diodes: 8x8 R grid (100..10k log-uniform) + 16 diodes (IS=1e-14, N=1, RS=10), "
                       "V source at the corner swept 0..5 V in 256 points, independent points from 0 V, plain FP64",
           "lanes": int(values.shape[0]), "unknowns": int(fr.n), "seed": seed,
           "l2": "flushed between timed steps (256 MiB write)", "reltol": 1e-3, "vntol": 1e-6}
    return fr, slots, values, cfg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sweep(fr, slots, values, threads):
    """The oracle's per-point solves on `threads` host threads (ctypes calls
    release the GIL), each worker taking the next chunk of points."""
    from oracle import oracle
    chunks = np.array_split(np.arange(values.shape[0]), max(1, threads * 4))
    warm = np.zeros(fr.n)
    conv = 0

    def run(idx):
        if len(idx) == 0:
            return 0
        _, _, cv = oracle.dc_points(fr, slots, values[idx], warm=warm)
        return int(cv.sum())

    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        for c in ex.map(run, chunks):
            conv += c
    return conv


def reference_arm(args, rank, world):
    if rank != 0:
        return
    fr, slots, values, cfg = workload()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sweep(fr, slots, values, threads)
    t0 = time.perf_counter()
    pts = 0
    for _ in range(args.steps):
        pts += cpu_sweep(fr, slots, values, threads)
    dt = time.perf_counter() - t0
    v = pts / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} batches of {values.shape[0]} points"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def algorithmic_bytes(fr, lanes_n, iters_total):
    """Bytes a lane-major, launch-per-phase design (the reference's) streams
    per Newton iteration and lane, by SURVEY's per-unit figures: eval reads x
    and writes the residual and matrix, the refactor reads A and writes
    L, U and the diagonal, the solve reads them and rhs and writes dx."""
    from oracle import oracle
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rc, tape = oracle.factor_tape(n, cp, ri, np.ones(nnz) + np.eye(1, nnz, 0).ravel())
    nlu = len(tape["li"]) + len(tape["ui"])
    per_iter = 8 * (n + nnz + n) + 8 * (nnz + nlu + n) + 8 * (nlu + n + n + n)
    return per_iter * iters_total


def fused_hbm_bytes(fr, rec_size, lanes_n):
    """HBM bytes the fused kernel must move per solve: each lane's records and
    start point in, its solution, iteration count and status out."""
    return lanes_n * (8 * rec_size + 8 * fr.n * 2 + 8)


def lu_replay_roofline(fr, ctx, hbm_peak, peak_src, lanes_n=32768, reps=5):
    """The standalone lane refactor + solve kernel (the reference's
    arp_lane_refactor + arp_lane_solve) over a batch larger than L2: A and
    rhs in, the L/U/diagonal tape values and dx out, per lane."""
    import torch
    from oracle import oracle
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(7)
    lead = rng.uniform(0.5, 2.0, nnz)
    for j in range(n):
        lead[cp[j] + np.searchsorted(ri[cp[j]:cp[j + 1]], j)] += 8.0
    a = torch.tensor(lead, dtype=torch.float64, device="cuda").repeat(lanes_n, 1)
    a *= torch.empty_like(a).uniform_(0.9, 1.1)
    rhs = torch.randn((lanes_n, n), dtype=torch.float64, device="cuda")
    dx = torch.empty_like(rhs)
    bad = torch.zeros(lanes_n, dtype=torch.uint8, device="cuda")
    ctx.lu_replay(lead, a.data_ptr(), rhs.data_ptr(), dx.data_ptr(), bad.data_ptr(), 1)
    nu, nl, ntv = ctx.tape_size()
    tv = torch.empty((lanes_n, ntv), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps + 2):
        torch.cuda.synchronize()
        ms.append(ctx.lu_replay(lead, a.data_ptr(), rhs.data_ptr(), dx.data_ptr(), bad.data_ptr(),
                                lanes_n, tv.data_ptr()))
    t = float(np.mean(ms[2:])) / 1e3
    per_lane = 8 * (nnz + n) + 8 * (ntv - 1 + n) + 1
    achieved = lanes_n * per_lane / t / 1e9
    return {"kernel": "lu_replay_kernel", "lanes": lanes_n, "ms": t * 1e3,
            "bytes_per_lane": per_lane, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "peak_source": peak_src,
            "bad_lanes": int(bad.sum().item())}


def our_arm(args, rank, world):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from espice_b200 import lanes
    fr, slots, values, cfg = workload(seed=1)
    ctx = lanes.DcLanes(fr, device=local)
    ctx.set_lanes(slots, values)
    N, n = values.shape[0], fr.n
    d_x0 = torch.zeros((N, n), dtype=torch.float64, device="cuda")
    d_x = torch.zeros_like(d_x0)
    d_it = torch.zeros(N, dtype=torch.int32, device="cuda")
    d_st = torch.zeros(N, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    opts = lanes.newton_opts()

    def step():
        d_x.copy_(d_x0)
        torch.cuda.synchronize()
        return ctx.solve_device(d_x.data_ptr(), d_it.data_ptr(), d_st.data_ptr(), cold=False, opts=opts)

    for _ in range(args.warmup):
        step()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ms, launches, conv, iters, peeled = [], 0, 0, 0, 0
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            s = step()
            ms.append(s["kernel_ms"])
            launches += s["launches"]
            conv += s["converged"]
            peeled += s["peeled"]
            iters += int(d_it.sum().item())
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    dev_s = sum(ms) / 1e3

    # e2e through the public API with host buffers (pinned), copies included.
    x0_h = torch.zeros((N, n), dtype=torch.float64).pin_memory().numpy()
    e2e_t = []
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        xh, ith, sth, _ = ctx.solve(x0=x0_h, opts=opts)
        t2 = time.perf_counter()
        if i >= args.warmup:
            e2e_t.append(t2 - t1)
    e2e_s = sum(e2e_t)
    e2e_conv = int((sth == lanes.LANE_CONVERGED).sum()) * args.steps

    # max over ranks
    if world > 1:
        t = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dev_s, e2e_s = float(t[0]), float(t[1])
        c = torch.tensor([conv, e2e_conv], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(c)
        conv, e2e_conv = int(c[0]), int(c[1])
    if rank != 0:
        ctx.close()
        return

    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    per_launch_ms = sum(ms) / max(1, launches)
    achieved = fused_hbm_bytes(fr, lanes.record_size(fr), N) / (sum(ms) / args.steps / 1e3) / 1e9
    alg = algorithmic_bytes(fr, N, iters / args.steps)
    out = {
        "metric": METRIC, "value": conv / dev_s, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "e2e": {"value": e2e_conv / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": int(N * n * 8),
                "d2h_bytes_per_step": int(N * n * 8 + 2 * N * 4)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": None,
                     "peak_source": peak_src,
                     "note": "fused dc_newton_kernel: unavoidable HBM bytes (records, start point, "
                             "solution) per launch / device time; the Newton working set stays in "
                             "shared memory, so the kernel is latency-bound, not HBM-bound",
                     "alg_bytes_lane_major_per_step": alg,
                     "alg_equivalent_gbs": alg / (sum(ms) / args.steps / 1e3) / 1e9},
        "newton_iters_per_point": iters / max(1, args.steps * N),
        "peeled_lanes": peeled, "clocks": clk.summary(), "wall_s_timed": wall,
    }
    out["lu_roofline"] = lu_replay_roofline(fr, ctx, hbm_peak, peak_src)
    if args.cpu_baseline:
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        pts = 0
        reps = 0
        while time.perf_counter() - t0 < args.cpu_seconds:
            pts += cpu_sweep(fr, slots, values, threads)
            reps += 1
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": pts / dt, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{reps} batches of {N} points ({dt:.1f} s)"}
    print(json.dumps(out), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        backend = "nccl" if args.impl == "ours" else "gloo"
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        else:
            our_arm(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
