"""Benchmark: converged sweep points/s of the sweep-lane Newton path on B200,
learned warm start + mixed precision against plain FP64, at 1e-9.

    python bench.py --gpus N --steps K --warmup W [--impl reference]

Workload (one GPU): the 500-unknown BSIM3 analog block (498 unknowns with
ground, 120 MOSFETs: twenty five-transistor OTA followers on a 20 x 21 RC
mesh, a six-branch bias network and a source follower), 65,536 seeded sweep
points of its 16 parameters (two supplies, six bias currents 1-100 uA
log-uniform, temperature -40..125 C, seven VTO shifts of +-50 mV), each an
independent DC operating point solved to reltol 1e-9, vntol 1e-12 V, abstol
1e-15 A. A step is one pass over all 65,536 points:
- learned + mixed (`value`): the tanh MLP (16 -> 512 -> 512 -> 498, BF16
  tcgen05 GEMMs with FP32 accumulation, trained on the GPU on 32,768 other
  points' plain-solver solutions before timing) predicts every point's
  start; the mixed-precision block lanes (FP32 refactor and solves, FP64
  evaluation, residual, refinement and gates) run at most 8 Newton
  iterations from it; the points that did not converge are solved again from
  the nominal operating point;
- plain FP64 (`plain_fp64`): the FP64 block lanes from the nominal point.
`value` is converged points / device time (CUDA events around each step on
the launching stream, the lanes' records resident in HBM, L2 flushed before
each step). `e2e` is the same metric through the public API with host
buffers: each step uploads the points' parameter values (esl_set_lanes,
records derived on the device) and the network's inputs, and reads every
point's solution back. Side blocks: the 31-stage ring-oscillator transient
lanes (`ring_transient`), the grid-with-diodes DC sweep, sequential sweep
lanes, the ring's early-stopping period measure, the uneven batch of eight
topologies (plain and mixed) and the lane LU against the HBM roofline.
Under torchrun each rank runs its own points (independent seeds, no
collective on the data path, weak scaling); times are the max over ranks.

--impl reference times the reference's CPU algorithm on this host's cores
(the C restatement under oracle/, since the Zig reference cannot be built
here): plain FP64 Newton from the nominal operating point, one point per
worker thread, as the reference's sweep pool runs them.
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
RING_LANES = 1024


def workload(seed=1, lanes_n=RING_LANES, t_stop=None):
    from espice_b200 import decks
    fr, slots, values = decks.ring_oscillator(seed=seed, lanes=lanes_n)
    cfg = {"workload": "ring_oscillator: 31-stage CMOS ring, MOS1 (NMOS KP=120u VTO=0.45 LAMBDA=0.05; "
                       "PMOS KP=40u VTO=-0.45 LAMBDA=0.05; W/L=1u/0.18u), 10 fF per stage, VDD=1.8 V "
                       "(50 ps ramp), per-device VTO ~ N(nominal, 30 mV); trapezoidal to 20 ns, 1 ps "
                       "max step; a point = one lane's whole transient, plain FP64",
           "lanes": int(values.shape[0]), "unknowns": int(fr.n), "seed": seed,
           "t_stop": t_stop or decks.RING_T_STOP, "t_max": decks.RING_T_MAX,
           "l2": "flushed between timed steps (256 MiB write)", "reltol": 1e-3, "vntol": 1e-6}
    return fr, slots, values, cfg


def tran_opts_pair(t_stop=None):
    from espice_b200 import decks, lanes
    from oracle import oracle
    t_stop = t_stop or decks.RING_T_STOP
    return (lanes.tran_opts(t_stop, decks.RING_T_STEP, decks.RING_T_MAX),
            oracle.tran_opts(t_stop, decks.RING_T_STEP, decks.RING_T_MAX))


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


def cpu_tran(fr, slots, values, threads, seconds, keep=None):
    """The oracle's transient lanes on `threads` host threads (ctypes calls
    release the GIL), one lane per task, until `seconds` have passed (the
    lanes started by then finish). Returns (lanes done, wall seconds); with
    keep a dict, keep[lane] = (step statistics, final x) of each lane run."""
    from oracle import oracle
    _, oo = tran_opts_pair()
    done = 0
    t0 = time.perf_counter()

    def run(i):
        if time.perf_counter() - t0 > seconds:
            return 0
        _, _, _, st, x = oracle.tran(fr, slots, values[i:i + 1], oo)
        if keep is not None:
            keep[i] = (st[0].copy(), x[0].copy())
        return int(st[0, 0] == 0)

    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        for c in ex.map(run, range(values.shape[0])):
            done += c
    return done, time.perf_counter() - t0


def parity_block(keep, stats, x):
    """The GPU lanes (stats [lanes][8], x [lanes][n] of the e2e run) against
    the oracle's runs of the same lanes (keep, from the CPU baseline): how many
    lanes took every step decision the oracle took, and the largest deviation
    of their final solutions."""
    idx = sorted(keep)
    if not idx:
        return {"lanes": 0}
    so = np.stack([keep[i][0] for i in idx]).astype(np.int64)
    xo = np.stack([keep[i][1] for i in idx])
    sg = stats[idx].astype(np.int64)
    xg = x[idx]
    d = np.abs(xg - xo)
    scale = np.maximum(np.abs(xg), np.abs(xo))
    within = d <= 1e-12 + 1e-9 * scale
    rel = np.where(d > 1e-12, d / np.maximum(scale, 1e-300), 0.0)
    return {"lanes": len(idx), "decisions_equal": int((sg == so).all(axis=1).sum()),
            "bitwise_equal": int((xg.view(np.uint64) == xo.view(np.uint64)).all(axis=1).sum()),
            "within_tolerance": bool(within.all()), "max_abs_dev": float(d.max()),
            "max_rel_dev": float(rel.max()),
            "checked": "the step statistics (status, accepted, attempts, Newton iterations, Newton and LTE "
                       "rejections, breakpoint landings, operating-point iterations) and the final solution "
                       "of the lanes the CPU baseline ran, against the e2e run's; tolerance 1e-9 relative "
                       "or 1e-12 absolute"}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), for the baseline records."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


C4_POINTS = 65536
C4_TRAIN = 32768


def c4_workload(seed=2, points=C4_POINTS):
    """The metric's configuration: the analog block and `points` seeded
    points of its 16 parameters (seed 1 is the training set's)."""
    from espice_b200 import decks
    fr, expand = decks.analog_block()
    params, nominal = decks.analog_block_params(seed=seed, points=points)
    cfg = {"workload": "analog_block: 500-unknown BSIM3 analog block (498 unknowns incl. ground, 120 MOSFETs: "
                       "20 five-transistor OTA followers on a 20x21 RC mesh, a 6-branch bias network, a source "
                       "follower), 16 parameters (VDD, VREF, 6 bias currents 1-100 uA log-uniform, temperature "
                       "-40..125 C, 7 DELVTO shifts +-50 mV); a point = one independent DC operating point; "
                       "learned warm start + mixed-precision block lanes",
           "points": int(points), "unknowns": int(fr.n), "parameters": 16, "seed": seed,
           "training_points": C4_TRAIN, "training_seed": 1,
           "reltol": TIGHT["reltol"], "vntol": TIGHT["vntol"], "abstol": TIGHT["abstol"],
           "l2": "flushed before each timed step (256 MiB write); the lanes' records alone exceed L2"}
    return fr, expand, params, nominal, cfg


def cpu_dc(fr, slots, values, x0, opts, threads, seconds, keep=None):
    """The oracle's DC points (plain FP64 Newton from x0) on `threads` host
    threads (ctypes calls release the GIL), one point per task, until
    `seconds` have passed (the points started by then finish). Returns
    (converged points, wall seconds); with keep a dict, keep[i] = (x,
    iterations, converged) of each point run."""
    from oracle import oracle
    t0 = time.perf_counter()

    def run(i):
        if time.perf_counter() - t0 > seconds:
            return 0
        x, it, cv = oracle.dc_points(fr, slots, values[i:i + 1], warm=x0, opts=opts)
        if keep is not None:
            keep[i] = (x[0].copy(), int(it[0]), bool(cv[0]))
        return int(cv[0])

    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        done = sum(ex.map(run, range(values.shape[0])))
    return done, time.perf_counter() - t0


def reference_arm(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle
    fr, expand, params, nominal, cfg = c4_workload()
    oo = oracle.newton_opts(**TIGHT)
    xn, _, cvn = oracle.dc_points(fr, expand.slots, expand(nominal), warm=None, opts=oo)
    threads = os.cpu_count() or 1
    per_step = 128 * threads  # a bounded sample of the 65,536 points
    vals = expand(params[:per_step])
    for _ in range(args.warmup):
        cpu_dc(fr, expand.slots, vals[:threads], xn[0], oo, threads, 1e9)
    t0 = time.perf_counter()
    pts = 0
    for _ in range(args.steps):
        d, _ = cpu_dc(fr, expand.slots, vals, xn[0], oo, threads, 1e9)
        pts += d
    dt = time.perf_counter() - t0
    v = pts / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_model(),
                         "sample": f"{args.steps} steps of the first {per_step} of the {C4_POINTS} points, "
                                   "plain FP64 Newton from the nominal operating point"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# DRAM bytes per point of one mixed dc_block_kernel launch on the analog
# block, from an ncu capture (dram__bytes_read.sum + dram__bytes_write.sum,
# --set full) of a 4,096-point learned step: 419.1 MB read, 121.8 MB
# written. The kernel reads a point's records once and keeps its working set
# on chip, so the traffic grows with points, not with iterations.
C4_BLOCK_DRAM_BYTES_PER_LANE = (419.072256e6 + 121.783296e6) / 4096

# DRAM bytes per lane of one tran_kernel launch, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum, --set full) of 148 ring
# lanes to 0.1 ns: 1,478,144 B read, 0 B written. The kernel reads each
# lane's records once and keeps its working set in shared memory, so the
# traffic grows with lanes, not with simulated time.
TRAN_DRAM_BYTES_PER_LANE = 1478144 / 148


def lane_major_bytes(fr, nr_iters_total):
    """Bytes a lane-major, launch-per-phase design (the reference's GPU lanes)
    streams per Newton iteration and lane (the per-unit figures of the scope
    table): eval reads x and writes the residual and matrix, the refactor
    reads A and writes L, U and the diagonal, the solve reads them and rhs
    and writes dx."""
    from oracle import oracle
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    vals = np.ones(nnz)
    for j in range(n):
        vals[cp[j] + np.searchsorted(ri[cp[j]:cp[j + 1]], j)] += 8.0
    rc, tape = oracle.factor_tape(n, cp, ri, vals)
    nlu = len(tape["li"]) + len(tape["ui"])
    per_iter = 8 * (n + nnz + n) + 8 * (nnz + nlu + n) + 8 * (nlu + n + n + n)
    return per_iter * nr_iters_total


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
    return {"kernel": "lu_replay_kernel", "lanes": lanes_n, "unknowns": n, "ms": t * 1e3,
            "bytes_per_lane": per_lane, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
            "frac": achieved / hbm_peak, "peak_source": peak_src,
            "bad_lanes": int(bad.sum().item())}


def lu_lanes_roofline(fr, ctx, hbm_peak, peak_src, lanes_n=131072, reps=5):
    """The lane refactor + solve (one thread per lane, [entry][lane] planes:
    the reference's arp_lane_refactor + arp_lane_solve layout) over a batch
    far larger than L2: A and rhs in, the L/U/diagonal tape values and dx
    out. The headline figure is the tape compiled into code (lu_tape, built
    with NVRTC on the first call); the interpreted lane kernel, bitwise the
    same, is timed beside it."""
    import torch
    from oracle import oracle
    cp, ri = oracle.pattern(fr)
    n, nnz = fr.n, len(ri)
    rng = np.random.default_rng(7)
    lead = rng.uniform(0.5, 2.0, nnz)
    for j in range(n):
        lead[cp[j] + np.searchsorted(ri[cp[j]:cp[j + 1]], j)] += 8.0
    a = torch.tensor(lead, dtype=torch.float64, device="cuda")[:, None].repeat(1, lanes_n)
    a *= torch.empty_like(a).uniform_(0.9, 1.1)
    rhs = torch.randn((n, lanes_n), dtype=torch.float64, device="cuda")
    dx = torch.empty_like(rhs)
    bad = torch.zeros(lanes_n, dtype=torch.uint8, device="cuda")
    ctx.lu_lanes(lead, a.data_ptr(), rhs.data_ptr(), dx.data_ptr(), bad.data_ptr(), 32)
    nu, nl, ntv = ctx.tape_size()
    tv = torch.empty((ntv, lanes_n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps + 2):
        torch.cuda.synchronize()
        ms.append(ctx.lu_lanes(lead, a.data_ptr(), rhs.data_ptr(), dx.data_ptr(), bad.data_ptr(), lanes_n,
                               tv.data_ptr()))
    t_int = float(np.mean(ms[2:])) / 1e3
    per_lane = 8 * (nnz + n) + 8 * (ntv - 1 + n) + 1
    # the compiled tape on the same lanes, checked bitwise against the
    # interpreted kernel
    dxc, tvc = torch.empty_like(dx), torch.empty_like(tv)
    badc = torch.zeros_like(bad)
    msc = []
    for _ in range(reps + 2):
        torch.cuda.synchronize()
        msc.append(ctx.lu_lanes_compiled(lead, a.data_ptr(), rhs.data_ptr(), dxc.data_ptr(), badc.data_ptr(),
                                         lanes_n, tvc.data_ptr()))
    t = float(np.mean(msc[2:])) / 1e3
    achieved = lanes_n * per_lane / t / 1e9
    log = ctx.lu_compiled_log()
    out = {"kernel": "lu_tape (the pivot tape compiled with NVRTC)", "lanes": lanes_n, "unknowns": n,
           "ms": t * 1e3, "bytes_per_lane": per_lane, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
           "frac": achieved / hbm_peak, "peak_source": peak_src, "bad_lanes": int(badc.sum().item()),
           "bitwise_vs_interpreted": bool(torch.equal(dxc.view(torch.int64), dx.view(torch.int64))
                                          and torch.equal(tvc[:ntv - 1].view(torch.int64),
                                                          tv[:ntv - 1].view(torch.int64))),
           "ptxas": " ".join(x.strip() for x in log.splitlines() if "registers" in x or "spill" in x),
           "interpreted": {"kernel": "lu_lanes_kernel", "ms": t_int * 1e3,
                           "achieved": lanes_n * per_lane / t_int / 1e9,
                           "frac": lanes_n * per_lane / t_int / 1e9 / hbm_peak}}
    # mixed precision (FP32 factors, FP64 refinement) on the same lanes: A and
    # rhs in, dx out (refinement re-reads are its own cost, not counted)
    dxm = torch.empty_like(rhs)
    refine = torch.zeros(lanes_n, dtype=torch.uint8, device="cuda")
    msm = []
    for _ in range(reps + 2):
        torch.cuda.synchronize()
        msm.append(ctx.lu_lanes_mixed(lead, a.data_ptr(), rhs.data_ptr(), dxm.data_ptr(), bad.data_ptr(), lanes_n,
                                      refine.data_ptr()))
    tm = float(np.mean(msm[2:])) / 1e3
    rel = float(((dxm - dx).abs() / dx.abs().clamp_min(1e-300)).max())
    # the mixed form compiled into code, on the same lanes
    dxc2 = torch.empty_like(rhs)
    msc2 = []
    for _ in range(reps + 2):
        torch.cuda.synchronize()
        msc2.append(ctx.lu_lanes_mixed_compiled(lead, a.data_ptr(), rhs.data_ptr(), dxc2.data_ptr(), bad.data_ptr(),
                                                lanes_n, refine.data_ptr()))
    tmc = float(np.mean(msc2[2:])) / 1e3
    out["mixed_compiled"] = {"kernel": "lu_tape_mixed (FP32 factors in registers, FP64 refinement, NVRTC)",
                             "ms": tmc * 1e3, "speedup_vs_fp64_compiled": t / tmc,
                             "achieved_gbs": lanes_n * 8 * (nnz + 2 * n) / tmc / 1e9,
                             "mean_corrections": float(refine.double().mean()),
                             "max_rel_dev_vs_fp64": float(((dxc2 - dx).abs() / dx.abs().clamp_min(1e-300)).max())}
    out["mixed"] = {"kernel": "lu_lanes_mixed_kernel", "ms": tm * 1e3, "speedup_vs_fp64": t / tm,
                    "bytes_per_lane": 8 * (nnz + 2 * n), "achieved_gbs": lanes_n * 8 * (nnz + 2 * n) / tm / 1e9,
                    "mean_corrections": float(refine.double().mean()), "max_rel_dev_vs_fp64": rel}
    return out


def dc_grid_diodes(args, local, flush):
    """The DC sweep of the grid-with-diodes deck (256 independent points from
    0 V, one fused DC launch per step), device-timed and end to end."""
    import torch
    from espice_b200 import decks, lanes
    fr, slots, values = decks.grid_diodes(seed=1, points=256)
    ctx = lanes.DcLanes(fr, device=local)
    ctx.set_lanes(slots, values)
    N, n = values.shape[0], fr.n
    d_x = torch.zeros((N, n), dtype=torch.float64, device="cuda")
    d_it = torch.zeros(N, dtype=torch.int32, device="cuda")
    d_st = torch.zeros(N, dtype=torch.int32, device="cuda")
    opts = lanes.newton_opts()
    ms, conv = [], 0
    for i in range(args.warmup + args.steps):
        d_x.zero_()
        flush.zero_()
        torch.cuda.synchronize()
        s = ctx.solve_device(d_x.data_ptr(), d_it.data_ptr(), d_st.data_ptr(), cold=False, opts=opts)
        if i >= args.warmup:
            ms.append(s["kernel_ms"])
            conv += s["converged"]
    x0_h = torch.zeros((N, n), dtype=torch.float64).pin_memory().numpy()
    e2e_t, e2e_conv = [], 0
    for i in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        _, _, sth, _ = ctx.solve(x0=x0_h, opts=opts)
        t2 = time.perf_counter()
        if i >= args.warmup:
            e2e_t.append(t2 - t1)
            e2e_conv += int((sth == lanes.LANE_CONVERGED).sum())
    # the warp lanes' device-buffer result of the timed steps (from 0 V)
    d_x.zero_()
    ctx.solve_device(d_x.data_ptr(), d_it.data_ptr(), d_st.data_ptr(), cold=False, opts=opts)
    x_fp64 = d_x.cpu().numpy()
    it_fp64 = d_it.cpu().numpy()
    ctx.close()
    # the same points in mixed precision (the block lanes: FP32 refactor and
    # solves, every Newton step refined in FP64 to 1e-12 of the residual)
    mx = lanes.DcLanes(fr, device=local)
    mx.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK)
    mx.set_lanes(slots, values)
    mms, mconv = [], 0
    for i in range(args.warmup + args.steps):
        d_x.zero_()
        flush.zero_()
        torch.cuda.synchronize()
        s = mx.solve_device(d_x.data_ptr(), d_it.data_ptr(), d_st.data_ptr(), cold=False, opts=opts)
        if i >= args.warmup:
            mms.append(s["kernel_ms"])
            mconv += s["converged"]
    dev, within = _dev(d_x.cpu().numpy(), x_fp64)
    same_it = int((d_it.cpu().numpy() == it_fp64).sum())
    mx.close()
    return {"workload": "grid_diodes: 8x8 R grid (100..10k log-uniform) + 16 diodes (IS=1e-14, N=1, "
                        "RS=10), source swept 0..5 V in 256 independent points from 0 V",
            "value": conv / (sum(ms) / 1e3), "unit": UNIT, "ms_per_step": float(np.mean(ms)),
            "e2e": conv and e2e_conv / sum(e2e_t),
            "mixed_block_lanes": {"value": mconv / (sum(mms) / 1e3), "ms_per_step": float(np.mean(mms)),
                                  "over_fp64_warp_lanes": (mconv / sum(mms)) / (conv / sum(ms)),
                                  "max_rel_dev_vs_fp64": dev, "within_1e-9_rel_or_1e-12_abs": within,
                                  "iterations_equal_fp64": same_it}}


def dc_sweep_lanes(args, local, flush):
    """Sequential .dc sweeps, one per lane: 1024 Monte-Carlo samples of the
    grid-with-diodes deck (four grid resistors scaled by exp(U(-0.5, 0.5)) per
    sample), each sweeping its source 0..5 V in 256 points as dc.zig does
    (predictor, limiting against the last point, warm Newton, cold rung on
    failure), all in one launch."""
    from espice_b200 import decks, lanes
    from espice_b200.circuit import R, V
    fr, _, _ = decks.grid_diodes(seed=1, points=4)
    rs = fr.slots_of(R, "r")[:4]
    nominal = np.array([fr.param(s) for s in rs])
    rng = np.random.default_rng(11)
    lane_vals = nominal * np.exp(rng.uniform(-0.5, 0.5, size=(1024, len(rs))))
    src = fr.slots_of(V, "dc")[0]
    pts = np.linspace(0.0, 5.0, 256)
    ctx = lanes.DcLanes(fr, device=local)
    ctx.set_lanes(rs, lane_vals)
    ms, conv, left = [], 0, 0
    for i in range(args.warmup + args.steps):
        flush.zero_()
        x, it, cv, st, t = ctx.sweep(src, pts)
        if i >= args.warmup:
            ms.append(t)
            conv += int(cv.sum())
            left += int((st != lanes.SWEEP_DONE).sum())
    ctx.close()
    return {"workload": "grid_diodes sweep lanes: 1024 samples x 256 sequential points (0..5 V)",
            "value": conv / (sum(ms) / 1e3), "unit": UNIT, "ms_per_step": float(np.mean(ms)),
            "lanes_left_tape": left, "newton_iters_per_point": float(it.mean())}


def ring_period_early_stop(args, local, flush):
    """The ring oscillator's period as a streamed measure (TRIG v(s0) VAL=0.9
    RISE=2, TARG v(s0) VAL=0.9 RISE=3) on the headline's 1024 lanes and
    20 ns window, each lane ending its transient once the card resolves
    (tran.zig's early stop). Lanes/s counts lanes that resolved."""
    from espice_b200 import decks, lanes
    fr, slots, values = decks.ring_oscillator(lanes=1024)
    s0 = fr.unknown("v(s0)")
    card = [lanes.trig_targ(lanes.meas_clause(s0, val=0.9, rise=2), lanes.meas_clause(s0, val=0.9, rise=3))]
    t_stop = args.t_stop or decks.RING_T_STOP
    o = lanes.tran_opts(t_stop, decks.RING_T_STEP, decks.RING_T_MAX, max_steps=10_000_000)
    ctx = lanes.DcLanes(fr, device=local)
    ctx.set_lanes(slots, values)
    ms, resolved, steps = [], 0, 0
    for i in range(min(args.warmup, 1) + max(1, args.steps // 5)):
        flush.zero_()
        v, st, _, t = ctx.tran_meas(o, card, early_stop=True)
        if i >= min(args.warmup, 1):
            ms.append(t)
            resolved += int((st[:, 0] == lanes.TRAN_RESOLVED).sum())
            steps += int(st[:, 1].sum())
    ctx.close()
    n = len(ms)
    return {"workload": "ring_oscillator period measure with early stop: 1024 lanes, t_stop %g s" % t_stop,
            "value": resolved / (sum(ms) / 1e3), "unit": "measured lanes/s", "ms_per_step": float(np.mean(ms)),
            "resolved_fraction": resolved / (n * 1024), "accepted_steps_per_lane": steps / (n * 1024),
            "period_s_median": float(np.nanmedian(v[:, 0]))}


# The accuracy setting of the metric's configurations: Newton stops when a
# step is below 1e-9 of the unknown (and 1e-12 V / 1e-15 A), so every start
# converges to the same solution within the parity tolerance (at reltol 1e-3
# a point's result depends on its start at the 1e-3 level).
TIGHT = dict(reltol=1e-9, vntol=1e-12, abstol=1e-15)
# Mixed precision refines the Newton steps within this many tolerances of
# convergence (esl_solve_mode.refine_skip); the steps farther out go
# unrefined, their FP32 error corrected by the iterations after them.
REFINE_SKIP = 1e3


def _dev(a, b):
    """(max relative deviation of a from b, fraction of points within 1e-9
    relative or 1e-12 absolute on every unknown)."""
    d = np.abs(a - b)
    scale = np.maximum(np.abs(a), np.abs(b))
    rel = np.where(d > 1e-12, d / np.maximum(scale, 1e-300), 0.0)
    within = np.all(d <= 1e-12 + 1e-9 * scale, axis=1)
    return float(rel.max()), float(within.mean())


def uneven_c3(args, local, flush, lanes_per_topo=512):
    """Uneven batching on its configuration: 4,096 DC lanes over the eight
    mesh-with-gates topologies (50 to 2,000 unknowns, 512 supply values each
    in [0.8, 1.8] V) in one launch of the block lanes, cold starts, plain FP64
    against mixed precision (refinement to 1e-12 of the residual), every step
    refined and, as the headline's mixed form, only the steps within
    REFINE_SKIP tolerances of convergence."""
    import torch
    from espice_b200 import decks, lanes
    from oracle import oracle
    sizes = decks.MESH_GATES_SIZES
    vals = np.linspace(0.8, 1.8, lanes_per_topo).reshape(-1, 1)
    out = {"workload": "mesh_gates: 8 seeded topologies of " + ", ".join(str(s) for s in sizes) +
                       f" unknowns (RC mesh + BSIM3 INV/NAND2), {lanes_per_topo} supply values each, one launch",
           "newton": "reltol 1e-3, vntol 1e-6 (the deck defaults), cold starts"}
    res = {}
    for prec, name, skip in ((lanes.PREC_FP64, "fp64", 0.0), (lanes.PREC_MIXED, "mixed", 0.0),
                             (lanes.PREC_MIXED, "mixed_skip", REFINE_SKIP)):
        ctxs, bufs = [], []
        for sz in sizes:
            fr, slots = decks.mesh_gates(sz)
            c = lanes.DcLanes(fr, device=local)
            c.set_mode(precision=prec, path=lanes.PATH_BLOCK, refine_skip=skip)
            c.set_lanes(slots, vals)
            ctxs.append(c)
            bufs.append((torch.zeros((lanes_per_topo, fr.n), dtype=torch.float64, device="cuda"),
                         torch.zeros(lanes_per_topo, dtype=torch.int32, device="cuda"),
                         torch.zeros(lanes_per_topo, dtype=torch.int32, device="cuda")))
        times, conv = [], 0
        for i in range(2):
            flush.zero_()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            st = lanes.group_solve_device(ctxs, [b[0].data_ptr() for b in bufs], [b[1].data_ptr() for b in bufs],
                                          [b[2].data_ptr() for b in bufs], cold=[True] * len(ctxs))
            torch.cuda.synchronize()
            if i == 1:
                times.append(time.perf_counter() - t1)
                conv = sum(int((b[2] == lanes.LANE_CONVERGED).sum()) for b in bufs)
        res[name] = {"points_per_s": conv / times[0], "converged": conv, "device_ms": st[0]["kernel_ms"],
                     "x": [b[0].cpu().numpy() for b in bufs],
                     "refinements_per_lane": sum(s["refinements"] for s in st) / (lanes_per_topo * len(sizes))}
        for c in ctxs:
            c.close()
    out["plain_points_per_s"] = res["fp64"]["points_per_s"]
    out["mixed_points_per_s"] = res["mixed"]["points_per_s"]
    out["mixed_over_plain"] = res["mixed"]["points_per_s"] / res["fp64"]["points_per_s"]
    out["mixed_skip_points_per_s"] = res["mixed_skip"]["points_per_s"]
    out["mixed_skip_over_plain"] = res["mixed_skip"]["points_per_s"] / res["fp64"]["points_per_s"]
    out["device_ms"] = {k: res[k]["device_ms"] for k in res}
    out["refinements_per_lane"] = res["mixed"]["refinements_per_lane"]
    out["refinements_per_lane_skip"] = res["mixed_skip"]["refinements_per_lane"]
    devs, worst = [], 0.0
    for t, sz in enumerate(sizes):
        fr, slots = decks.mesh_gates(sz)
        idx = np.arange(0, lanes_per_topo, 128)
        xo, _, cvo = oracle.dc_points(fr, slots, vals[idx], warm=None)
        ok = cvo.astype(bool)
        dp, wp = _dev(res["fp64"]["x"][t][idx][ok], xo[ok])
        dm, wm = _dev(res["mixed"]["x"][t][idx][ok], xo[ok])
        ds, ws = _dev(res["mixed_skip"]["x"][t][idx][ok], xo[ok])
        worst = max(worst, dm, ds)
        devs.append({"unknowns": fr.n, "plain_vs_oracle": dp, "mixed_vs_oracle": dm, "mixed_within": wm,
                     "mixed_skip_vs_oracle": ds, "mixed_skip_within": ws})
    out["per_topology_max_rel_dev"] = devs
    out["mixed_max_rel_dev_vs_cpu_oracle"] = worst
    out["oracle_sample"] = "4 lanes per topology (every 128th)"
    return out


C5_LANES = 256
C5_WINDOW = 1e-10


def large_transient_c5(args, local):
    """The large transient configuration (C5): the 20,001-unknown digital
    block (500 BSIM3 NAND2 cells, 2,000 MOSFETs, on a planar RC mesh, 16
    seeded PWL pulse trains with 50 ps edges), 256 lanes with per-device
    DELVTO ~ N(0, 20 mV), trapezoidal, on the block lanes (a CTA per lane,
    the working set in the CTA's global slab). Timed over the first
    `c5_window` seconds of the 5 ns run with the 5 ns run's maximum step
    (10 ps), FP64 and mixed precision (FP32 refactor and solves, FP64
    refinement near convergence), each one persistent launch timed with CUDA
    events on the context's stream after a 2 ps warm-up run. The lanes'
    working sets (about 11 MB each) far exceed L2. The FP64 lanes' step
    decisions equal the oracle's (tests/test_gpu_block_tran.py); here the
    mixed lanes are checked against the FP64 lanes."""
    import torch
    from espice_b200 import decks, lanes
    fr, slots = decks.digital_block()
    N, n = args.c5_lanes, fr.n
    vals = decks.digital_block_vto(len(slots), N)
    go = lanes.tran_opts(args.c5_window, 1e-11, 1e-11, max_steps=100_000)
    warm = lanes.tran_opts(2e-12, 1e-11, 1e-11, max_steps=100_000)
    acc, nri = lanes.TS_FIELDS.index("accepted"), lanes.TS_FIELDS.index("nr_iters")
    res, info = {}, None
    for prec, name, skip in ((lanes.PREC_FP64, "fp64", 0.0), (lanes.PREC_MIXED, "mixed", REFINE_SKIP)):
        ctx = lanes.DcLanes(fr, device=local)
        ctx.set_mode(precision=prec, path=lanes.PATH_BLOCK, refine_skip=skip)
        ctx.set_lanes(slots, vals)
        d_x = torch.zeros((N, n), dtype=torch.float64, device="cuda")
        d_st = torch.zeros((N, len(lanes.TS_FIELDS)), dtype=torch.int32, device="cuda")
        ctx.tran_device(warm, d_x.data_ptr(), d_st.data_ptr())
        ms = ctx.tran_device(go, d_x.data_ptr(), d_st.data_ptr())
        st = d_st.cpu().numpy().astype(np.int64)
        corr = ctx.tran_refinements()
        if info is None:
            bi = ctx.block_info()
            info = {k: bi[k] for k in ("a_rows", "a_levels", "a_nops", "ntv", "lane_bytes", "in_smem", "ctas_per_sm")}
        ctx.close()
        done = int((st[:, 0] == lanes.TRAN_DONE).sum())
        steps = int(st[:, acc].sum())
        iters = int(st[:, nri].sum())
        res[name] = {"device_ms": ms, "lanes_done": done, "accepted_steps_per_lane": steps / N,
                     "newton_iters_per_lane": iters / N, "lane_steps_per_s": steps / (ms / 1e3),
                     "window_lanes_per_s": done / (ms / 1e3), "stats": st, "x": d_x.cpu().numpy()}
        if prec == lanes.PREC_MIXED:
            res[name]["refinements_per_newton_iter"] = corr / max(iters, 1)
    dev, within = _dev(res["mixed"]["x"], res["fp64"]["x"])
    same = int((res["mixed"]["stats"] == res["fp64"]["stats"]).all(axis=1).sum())
    for r in res.values():
        del r["stats"], r["x"]
    return {"workload": "digital_block: 20,001 unknowns (500 BSIM3 NAND2 cells = 2,000 MOSFETs on a planar RC "
                        "mesh, R 10-10k log-uniform, C 1-100 fF; 16 seeded PWL pulse trains, 50 ps edges), "
                        f"{N} lanes, per-device DELVTO ~ N(0, 20 mV), trapezoidal",
            "window_s": args.c5_window, "t_stop_config_s": 5e-9, "t_max_s": 1e-11, "lanes": N, "unknowns": n,
            "fp64": res["fp64"], "mixed": res["mixed"],
            "mixed_over_fp64": res["fp64"]["device_ms"] / res["mixed"]["device_ms"],
            "mixed_vs_fp64": {"max_rel_dev": dev, "within_1e-9_rel_or_1e-12_abs": within,
                              "lanes_with_equal_step_statistics": same},
            "block_lanes": info,
            "note": "a window of the 5 ns configuration (its whole run would hold the GPU for minutes); "
                    "lane_steps_per_s = accepted steps of all lanes / device time"}


def load_peaks():
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    return hbm_peak, "measured" if "hbm_gbs" in peaks else "fallback"


def ring_transient(args, rank, world, local, flush):
    """The transient Monte-Carlo lanes: the 31-stage MOS1 ring oscillator,
    1024 lanes, trapezoidal to 20 ns with a 1 ps maximum step; a point is one
    lane's whole transient, one tran_kernel launch per step. Device-timed,
    end to end (esl_set_lanes + esl_tran with host buffers), the CPU
    oracle's lanes/s on the host cores, and the lanes the CPU ran checked
    decision for decision against the e2e run."""
    import torch
    from espice_b200 import lanes, shard
    fr, slots, values, cfg = workload(seed=1 + rank, lanes_n=args.lanes, t_stop=args.t_stop)
    go, _ = tran_opts_pair(args.t_stop)
    ctx = lanes.DcLanes(fr, device=local)
    ctx.set_lanes(slots, values)
    N, n = values.shape[0], fr.n
    d_x = torch.zeros((N, n), dtype=torch.float64, device="cuda")
    d_st = torch.zeros((N, len(lanes.TS_FIELDS)), dtype=torch.int32, device="cuda")

    def step():
        torch.cuda.synchronize()
        return ctx.tran_device(go, d_x.data_ptr(), d_st.data_ptr())

    for _ in range(args.warmup):
        step()
    ms, done, steps_acc, nr_iters = [], 0, 0, 0
    ring_steps = max(1, args.steps // 2)
    for _ in range(ring_steps):
        flush.zero_()
        ms.append(step())
        st = d_st.cpu().numpy()
        done += int((st[:, 0] == lanes.TRAN_DONE).sum())
        steps_acc += int(st[:, 1].sum())
        nr_iters += int(st[:, 3].sum())
    dev_s = sum(ms) / 1e3
    e2e_t, e2e_done = [], 0
    for i in range(1 + ring_steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ctx.set_lanes(slots, values)
        _, _, _, sth, xh, _ = ctx.tran(go)
        t2 = time.perf_counter()
        if i >= 1:
            e2e_t.append(t2 - t1)
            e2e_done += int((sth[:, 0] == lanes.TRAN_DONE).sum())
    e2e_s = sum(e2e_t)
    dev_s, done = shard.reduce_run(dev_s, done)
    e2e_s, e2e_done = shard.reduce_run(e2e_s, e2e_done)
    if rank != 0:
        ctx.close()
        return None
    hbm_peak, peak_src = load_peaks()
    step_s = dev_s / ring_steps
    rec_bytes = lanes.record_size(fr) * 8
    hbm_bytes = N * (rec_bytes + 8 * n + 4 * len(lanes.TS_FIELDS))
    achieved = hbm_bytes / step_s / 1e9
    alg = lane_major_bytes(fr, nr_iters / ring_steps)
    out = {"config": cfg, "value": done / dev_s, "unit": "points/s (a point = one lane's whole transient)",
           "ms_per_step": 1e3 * step_s, "steps": ring_steps, "dtype": "f64",
           "e2e": {"value": e2e_done / e2e_s, "h2d_bytes_per_step": int(values.nbytes),
                   "d2h_bytes_per_step": int(N * n * 8 + N * 4 * len(lanes.TS_FIELDS))},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                        "frac": achieved / hbm_peak, "traffic": TRAN_DRAM_BYTES_PER_LANE * N,
                        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                          "tran_kernel launch on 148 ring lanes, scaled by lanes",
                        "peak_source": peak_src,
                        "note": "fused tran_kernel: unavoidable HBM bytes (records in, solution and step "
                                "statistics out) per launch / device time; every lane's working set stays in "
                                "shared memory for its whole transient (latency bound, not HBM bound)",
                        "alg_bytes_lane_major_per_step": alg, "alg_equivalent_gbs": alg / step_s / 1e9},
           "accepted_steps_per_point": steps_acc / max(1, ring_steps * N),
           "newton_iters_per_point": nr_iters / max(1, ring_steps * N)}
    out["lu_roofline"] = lu_lanes_roofline(fr, ctx, hbm_peak, peak_src)
    out["lu_roofline_warp_per_lane"] = lu_replay_roofline(fr, ctx, hbm_peak, peak_src)
    out["mixed_block_lanes_2ns"] = ring_mixed_window(fr, slots, values, local, 2e-9)
    if args.cpu_baseline:
        threads = os.cpu_count() or 1
        keep = {}
        d, dt = cpu_tran(fr, slots, values, threads, args.cpu_seconds, keep=keep)
        out["cpu_baseline"] = {"value": d / dt, "unit": "points/s", "cores": threads, "kind": "port",
                               "cpu": cpu_model(), "sample": f"{d} of the {N} lanes in {dt:.1f} s"}
        out["parity"] = parity_block(keep, sth, xh)
    ctx.close()
    return out


def ring_mixed_window(fr, slots, values, local, t_stop):
    """The ring's lanes in mixed precision (the block lanes: FP32 refactor
    and solves, every Newton step refined in FP64 to 1e-12 of the residual;
    the warp lanes are FP64 only) over the first t_stop of the run, against
    the FP64 warp lanes over the same window: device times of one launch
    each (CUDA events on the context's stream), the lanes whose step
    statistics are equal, and the end states' deviation."""
    import torch
    from espice_b200 import lanes
    go, _ = tran_opts_pair(t_stop)
    N, n = values.shape[0], fr.n
    res = {}
    for name, prec, path in (("fp64_warp", lanes.PREC_FP64, lanes.PATH_WARP),
                             ("mixed_block", lanes.PREC_MIXED, lanes.PATH_BLOCK)):
        ctx = lanes.DcLanes(fr, device=local)
        ctx.set_mode(precision=prec, path=path)
        ctx.set_lanes(slots, values)
        d_x = torch.zeros((N, n), dtype=torch.float64, device="cuda")
        d_st = torch.zeros((N, len(lanes.TS_FIELDS)), dtype=torch.int32, device="cuda")
        ctx.tran_device(tran_opts_pair(1e-11)[0], d_x.data_ptr(), d_st.data_ptr())
        ms = ctx.tran_device(go, d_x.data_ptr(), d_st.data_ptr())
        res[name] = (ms, d_st.cpu().numpy(), d_x.cpu().numpy(), ctx.tran_refinements())
        ctx.close()
    (mf, sf, xf, _), (mm, sm, xm, corr) = res["fp64_warp"], res["mixed_block"]
    dev, within = _dev(xm, xf)
    nr = int(sm[:, lanes.TS_FIELDS.index("nr_iters")].sum())
    return {"window_s": t_stop, "lanes": N, "fp64_warp_ms": mf, "mixed_block_ms": mm,
            "mixed_over_fp64": mf / mm, "lanes_with_equal_step_statistics": int((sm == sf).all(axis=1).sum()),
            "max_rel_dev_vs_fp64": dev, "within_1e-9_rel_or_1e-12_abs": within,
            "refinements_per_newton_iter": corr / max(nr, 1)}


def our_arm(args, rank, world):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    from espice_b200 import decks, lanes, learned, shard
    fr, expand, p_test, nominal, cfg = c4_workload(seed=2 + 2 * rank, points=args.points)
    cfg["training_points"] = args.train
    opts = lanes.newton_opts(**TIGHT)
    N, n = p_test.shape[0], fr.n
    slots = expand.slots
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    setup = {}

    # the nominal operating point (the plain path's start and the fallback's)
    plain = lanes.DcLanes(fr, device=local)
    plain.set_mode(precision=lanes.PREC_FP64, path=lanes.PATH_BLOCK)
    plain.set_lanes(slots, expand(nominal))
    x_nom = plain.solve(x0=None, opts=opts)[0][0]
    # the network, trained on the GPU on other points' plain-solver solutions
    t0 = time.perf_counter()
    p_train, _ = decks.analog_block_params(seed=1 + 2 * rank, points=args.train)
    plain.set_lanes(slots, expand(p_train))
    x_tr, _, st_tr, _ = plain.solve(x0=np.broadcast_to(x_nom, (args.train, n)), opts=opts)
    setup["training_solutions_s"] = time.perf_counter() - t0
    ok = st_tr == lanes.LANE_CONVERGED
    ws = learned.LearnedWarmStart(16, n, hidden=512, layers=3, device=local)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = ws.fit(p_train[ok], x_tr[ok], epochs=60, batch=256, lr=2e-3, lr_end=2e-5)
    torch.cuda.synchronize()
    setup["training_60_epochs_s"] = time.perf_counter() - t0
    vals = expand(p_test)
    t0 = time.perf_counter()
    plain.set_lanes(slots, vals)
    setup["set_lanes_s"] = time.perf_counter() - t0
    mixed = lanes.DcLanes(fr, device=local)
    mixed.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, refine_skip=REFINE_SKIP)
    mixed.set_lanes(slots, vals)
    fb = lanes.DcLanes(fr, device=local)
    fb.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, refine_skip=REFINE_SKIP)
    d_x = torch.empty((N, n), dtype=torch.float64, device="cuda")
    d_it = torch.zeros(N, dtype=torch.int32, device="cuda")
    d_st = torch.zeros(N, dtype=torch.int32, device="cuda")
    x_nom_d = torch.tensor(x_nom, device="cuda")
    d_p = torch.tensor(p_test, dtype=torch.float32, device="cuda")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        flush.zero_()
        torch.cuda.synchronize()
        ev0.record()
        r = fn()
        ev1.record()
        ev1.synchronize()
        return r, ev0.elapsed_time(ev1) / 1e3

    def learned_step(stats):
        return learned.solve(mixed, fb, ws, slots, vals, x_nom, k=8, opts=opts, d_values=d_p, stats_out=stats)

    def plain_step():
        d_x.copy_(x_nom_d.expand(N, n))
        return plain.solve_device(d_x.data_ptr(), d_it.data_ptr(), d_st.data_ptr(), cold=False, opts=opts)

    for _ in range(args.warmup):
        timed(lambda: learned_step([]))
        timed(plain_step)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    lt, lconv, lit, lfb, lstats = 0.0, 0, 0.0, 0, []
    # NVTX ranges mark the timed steps (a profiler can take its launch list
    # from them alone: ncu --nvtx --nvtx-include "learned_mixed_timed/")
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("learned_mixed_timed")
        for _ in range(args.steps):
            st_list = []
            (xl, it, conv, nfb), dt = timed(lambda: learned_step(st_list))
            lt += dt
            lconv += int(conv.sum())
            lit += float(it.mean())
            lfb += nfb
            lstats.append(st_list)
        torch.cuda.nvtx.range_pop()
        x_learned = xl.cpu().numpy()
        pt, pconv, pit, pstats = 0.0, 0, 0.0, []
        torch.cuda.nvtx.range_push("plain_fp64_timed")
        for _ in range(args.steps):
            sp, dt = timed(plain_step)
            pt += dt
            pconv += int((d_st == lanes.LANE_CONVERGED).sum())
            pit += float(d_it.double().mean())
            pstats.append(sp)
        torch.cuda.nvtx.range_pop()
    x_plain = d_x.cpu().numpy()
    it_plain = d_it.cpu().numpy().astype(np.int64)
    K = args.steps
    # attribution: the same learned + mixed steps refining every Newton step
    mixed.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK)
    fb.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK)
    at, aconv = 0.0, 0
    for _ in range(K):
        (_, _, conv, _), dt = timed(lambda: learned_step([]))
        at += dt
        aconv += int(conv.sum())
    mixed.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, refine_skip=REFINE_SKIP)
    fb.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, refine_skip=REFINE_SKIP)

    # e2e through the public API with host buffers: the points' parameters
    # in (the lanes' 16 live parameter values from pinned memory, expanded
    # to the 248 device fields on the device by esl_set_lanes_cols, and the
    # network's FP32 inputs), every point's solution out to pinned memory
    p_pin = torch.empty((N, p_test.shape[1]), dtype=torch.float32).pin_memory()
    lp_pin = torch.empty((N, p_test.shape[1]), dtype=torch.float64).pin_memory()
    x_host = torch.empty((N, n), dtype=torch.float64).pin_memory()
    d_p_e = torch.empty((N, p_test.shape[1]), dtype=torch.float32, device="cuda")
    e2e_t, e2e_conv, e2e_fb, h2d, d2h = 0.0, 0, 0, 0, 0
    for i in range(1 + K):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        lp = lp_pin.numpy()
        lp[:] = expand.lane_params(p_test)
        mixed.set_lanes(slots, lp, cols=expand.cols)
        p_pin.copy_(torch.from_numpy(p_test))
        d_p_e.copy_(p_pin)
        xl, it, conv, nfb = learned.solve(mixed, fb, ws, slots, lp, x_nom, k=8, opts=opts, d_values=d_p_e,
                                          cols=expand.cols)
        x_host.copy_(xl)
        t2 = time.perf_counter()
        if i >= 1:
            e2e_t += t2 - t1
            e2e_conv += int(conv.sum())
            e2e_fb += nfb
            h2d += lp.nbytes + p_pin.numel() * 4 + nfb * (lp.shape[1] + n) * 8
            d2h += N * n * 8 + 2 * N * 4 + nfb * n * 8

    # the mixed lanes' phase cycles (one untimed, profiled pass)
    mixed.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, profile=True, refine_skip=REFINE_SKIP)
    prof_stats = []
    learned_step(prof_stats)
    prof = mixed.block_profile()
    info = mixed.block_info()
    mixed.set_mode(precision=lanes.PREC_MIXED, path=lanes.PATH_BLOCK, refine_skip=REFINE_SKIP)

    lt, lconv = shard.reduce_run(lt, lconv)
    pt, pconv = shard.reduce_run(pt, pconv)
    e2e_t, e2e_conv = shard.reduce_run(e2e_t, e2e_conv)
    ring = ring_transient(args, rank, world, local, flush) if args.side else None
    if rank != 0:
        for c in (plain, mixed, fb):
            c.close()
        ws.close()
        return

    hbm_peak, peak_src = load_peaks()
    rec_bytes = lanes.record_size(fr) * 8
    lane_bytes = rec_bytes + 16 * n + 32  # records in, start in, solution out, lane words
    k_ms = lstats[-1][0]["kernel_ms"]
    achieved = N * lane_bytes / (k_ms / 1e3) / 1e9
    iters = max(prof["iterations"], 1)
    ref_per_iter = prof_stats[0]["refinements"] / iters
    at, aconv = shard.reduce_run(at, aconv)
    rows_per_iter = info["a_rows"] + info["b_rows"] + ref_per_iter * (info["f_rows"] + info["b_rows"])
    cyc = {k: prof[k] / iters for k in ("eval", "assemble", "refactor", "solve", "refine", "gates")}
    launches = sum(sum(x["launches"] + 1 for x in st) for st in lstats) + K * 10
    out = {
        "metric": METRIC, "value": lconv / lt, "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * lt / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic", "config": cfg,
        "e2e": {"value": e2e_conv / e2e_t, "unit": UNIT, "h2d_bytes_per_step": int(h2d / K),
                "d2h_bytes_per_step": int(d2h / K)},
        "gpu_launches": int(launches),
        "plain_fp64": {"value": pconv / pt, "unit": UNIT, "ms_per_step": 1e3 * pt / K,
                       "newton_iters_per_point": pit / K, "gpu_launches": int(sum(x["launches"] + 1 for x in pstats))},
        "learned_mixed_over_plain": (lconv / lt) / (pconv / pt),
        "mixed_refinement": {"refine_tol": 1e-12, "refine_skip": REFINE_SKIP,
                             "note": "FP32 refactor and solves; a Newton step whose FP32 solution is within "
                                     f"{REFINE_SKIP:g} tolerances of convergence is refined in FP64 on the residual "
                                     "to 1e-12 of it, a step farther out is taken as an inexact Newton step",
                             "refine_every_step_points_per_s": aconv / at,
                             "refinements_per_newton_iter": ref_per_iter},
        "newton_iters_per_point": lit / K, "fallback_points_per_step": lfb / K,
        "e2e_fallback_points_per_step": e2e_fb / K,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": C4_BLOCK_DRAM_BYTES_PER_LANE and
                     C4_BLOCK_DRAM_BYTES_PER_LANE * N,
                     "kernel": "dc_block_kernel (mixed precision, BSIM3): the learned step's Newton launch",
                     "kernel_ms": k_ms, "alg_bytes_per_lane": lane_bytes,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one mixed "
                                       "dc_block_kernel launch on a reduced point count, scaled by points",
                     "peak_source": peak_src,
                     "note": "each lane's working set stays in its CTA's shared memory for the whole solve, so "
                             "HBM carries only records, starts and solutions: the kernel is bound by the "
                             "latency of its dependent program rows (the latency block)"},
        "latency": {"cycles_per_newton_iter": {k: round(v) for k, v in cyc.items()},
                    "rows_per_newton_iter": rows_per_iter,
                    "refactor_cycles_per_row": cyc["refactor"] / info["a_rows"],
                    "program_a": {"rows": info["a_rows"], "dependency_levels": info["a_levels"],
                                  "ops": info["a_nops"], "levels_over_rows": info["a_levels"] / info["a_rows"]},
                    "program_b_rows": info["b_rows"], "program_f_rows": info["f_rows"],
                    "refinements_per_newton_iter": ref_per_iter,
                    "ctas_per_sm": info["ctas_per_sm"], "lane_bytes": info["lane_bytes"],
                    "note": "cycles of one CTA (one lane) per Newton iteration by phase, thread 0's clock64; "
                            "rows are CTA-wide steps of the tape programs, each ending in a barrier; "
                            "levels_over_rows: the dependency bound of program A over its scheduled rows"},
        "setup": dict(setup, train_loss_first_last=[float(loss[0]), float(loss[-1])]),
        "clocks": clk.summary(),
    }
    if args.cpu_baseline:
        from oracle import oracle
        oo = oracle.newton_opts(**TIGHT)
        xo_nom, _, _ = oracle.dc_points(fr, slots, expand(nominal), warm=None, opts=oo)
        threads = os.cpu_count() or 1
        keep = {}
        d, dt = cpu_dc(fr, slots, vals, xo_nom[0], oo, threads, args.cpu_seconds, keep=keep)
        out["cpu_baseline"] = {"value": d / dt, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_model(),
                               "sample": f"the first {len(keep)} of the {N} points in {dt:.1f} s, plain FP64 "
                                         "Newton from the nominal operating point, one point per thread"}
        idx = np.array(sorted(keep), dtype=np.int64)
        xo = np.stack([keep[i][0] for i in idx])
        ito = np.array([keep[i][1] for i in idx])
        cvo = np.array([keep[i][2] for i in idx])
        dp = _dev(x_plain[idx][cvo], xo[cvo])
        dl = _dev(x_learned[idx][cvo], xo[cvo])
        out["parity"] = {
            "points": int(len(idx)), "oracle_converged": int(cvo.sum()),
            "plain_fp64": {"bitwise_equal": int((x_plain[idx].view(np.uint64) == xo.view(np.uint64)).all(1).sum()),
                           "iterations_equal": int((it_plain[idx] == ito).sum()), "max_rel_dev": dp[0]},
            "learned_mixed": {"max_rel_dev": dl[0], "within_1e-9_rel_or_1e-12_abs": dl[1]},
            "checked": "every point the CPU baseline solved: the plain FP64 lanes' solution bitwise and their "
                       "Newton iteration count against the oracle's; the learned + mixed lanes' solution within "
                       "1e-9 relative or 1e-12 absolute of it"}
    out["learned_vs_plain_points_all"] = dict(zip(("max_rel_dev", "within_1e-9"), _dev(x_learned, x_plain)))
    for c in (plain, mixed, fb):
        c.close()
    ws.close()
    if args.side:
        out["ring_transient"] = ring
        out["dc_grid_diodes"] = dc_grid_diodes(args, local, flush)
        out["dc_sweep_lanes"] = dc_sweep_lanes(args, local, flush)
        out["ring_period_early_stop"] = ring_period_early_stop(args, local, flush)
        out["uneven_c3"] = uneven_c3(args, local, flush)
        # one GPU's measurement: under torchrun the other ranks wait at the
        # closing barrier meanwhile, so it runs only at N = 1
        if args.c5_window > 0 and world == 1:
            out["large_transient_c5"] = large_transient_c5(args, local)
    print(json.dumps(out), flush=True)




def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    # a reduced case for profiler captures (the benchmark itself uses the defaults)
    ap.add_argument("--lanes", type=int, default=RING_LANES)
    ap.add_argument("--points", type=int, default=C4_POINTS)
    ap.add_argument("--train", type=int, default=C4_TRAIN)
    ap.add_argument("--no-side", dest="side", action="store_false")
    ap.add_argument("--t-stop", type=float, default=None)
    ap.add_argument("--c5-window", type=float, default=C5_WINDOW, help="seconds of the C5 run to time (0: skip)")
    ap.add_argument("--c5-lanes", type=int, default=C5_LANES)
    # the C5 block alone (a small case for a profiler capture of its kernel)
    ap.add_argument("--only-c5", action="store_true")
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
        if args.only_c5:
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            print(json.dumps(large_transient_c5(args, int(os.environ.get("LOCAL_RANK", "0")))), flush=True)
        elif args.impl == "reference":
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
