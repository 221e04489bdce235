"""Benchmark: explicit MPM particle-steps/s on the B200.

Workload (default): the 3D granular column collapse -- 200x100x50 hex8 cells
of 0.01 m, MohrCoulomb (E=1e7, nu=0.3, phi=30, c=0, psi=0, rho=1800), USL,
FLIP, frictional floor mu=0.4, dt=2e-6, 2x2x2 particles per cell in the block
[0,1]x[0,1]x[0,0.5] (4,000,000 particles), K0 geostatic initial stress.
Synthetic seeded inputs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision mixed|fp64]

One JSON line on stdout (rank 0).  ``value`` is device-timed (CUDA events on
the solver's stream, state resident in HBM) for the chosen precision (mixed by
default); ``fp64`` holds the FP64 path timed on the same workload and steps and
the mixed path's per-field deviation from it; ``accuracy`` gives that deviation
at fixed step counts (50, 500, 2000 by default) beside the FP64 path's own
one-ulp floor, and ``late`` a second timed window after them; ``persistent``
times the one-launch persistent form of the same step; ``e2e`` goes through the
public API with page-locked host arrays (load -> K steps -> read back);
``roofline`` reports the dominant kernel's algorithmic bytes per launch over its
event-timed average duration, and ``roofline.step`` the whole step's bytes per
particle-step times the throughput; ``cpu_baseline`` times the CPU oracle on a
bounded sample.
Under torchrun (N>1) every rank runs an independent replica (weak scaling; one
run cut into slabs over several GPUs is mpm_b200.slab, not timed here), timing
is the max over ranks.
"""
import argparse
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic bytes per particle of the particle kernels, MohrCoulomb USL
# (compulsory particle-state traffic: every field read once, every field the
# kernel changes written once; nodal gathers hit L2 and are not counted).
BYTES_PER_PARTICLE = {
    ("fp64", 3): {
        # read x u v 72, stress strain 96, F 72, volume density 16, cell 4,
        # material 2, constraint slot 2, MC state 72
        "g2p": 336 + 296,   # write x u v stress strain F V rho 256, MC state that changes 40
        "p2g": 116,         # read x 24, v 24, mass 8, stress 48, volume 8, order 4
    },
    ("mixed", 3): {
        # read x u 48 (FP64), v stress strain H V0 rho0 P 108 (FP32), MC state
        # 32, cell material slot 8; write x u 48, v stress strain H P 100, MC 16
        "g2p": 196 + 164,
        "p2g": 68,          # read x 24, v 12, mass 4, stress 24, V0 P 8 (FP32)
    },
    ("fp64", 2): {
        # read x u v 48, stress 32, strain 24, F 32, V rho 16, MC 72, slots 8;
        # write the first 152 + MC that changes 40
        "g2p": 232 + 192,
        "p2g": 84,
    },
    ("mixed", 2): {
        # read x u 32, v stress strain H V0 rho0 P 64, MC 32, slots 8; write
        # x u 32, v stress strain H P 56, MC 16
        "g2p": 136 + 104,
        "p2g": 52,
    },
}
# DRAM traffic per particle of the particle kernels as ncu measured it
# (dram__bytes_read.sum + dram__bytes_write.sum of one launch, USL MohrCoulomb
# column of 1,000,000 particles, step 3), scaled by the particles of a launch
# for the roofline's "traffic": the 4M-particle launch is too large for a
# multi-pass capture.
MEASURED_TRAFFIC_PER_PARTICLE = {
    ("mixed", 3): {"g2p": 329.7, "p2g": 117.0},
    ("fp64", 3): {"g2p": 615.4, "p2g": 186.3},
}
# Algorithmic bytes per particle-step of the whole step (compulsory particle-state
# traffic plus one write and one read of each nodal field per active node), for
# the step-level roofline.  3D MohrCoulomb: FP64 576 particle + 26 grid, mixed
# 340 + 20.  2D MohrCoulomb: mixed 276 + 25; FP64 reads x u v stress strain F
# V rho m pdstrain (21 doubles) and the cell, writes 25 doubles and the cell
# (376) + 25 grid.
STEP_BYTES_PER_PARTICLE = {("fp64", 3): 602, ("mixed", 3): 360, ("fp64", 2): 401,
                           ("mixed", 2): 301}
DTYPES = {"fp64": "f64", "mixed": "f32+f64"}
FIELDS = ("u", "v", "stress", "strain", "F", "volume", "density")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--block", default="100,100,50", help="particle block in cells")
    ap.add_argument("--workload", default="column",
                    choices=["column", "footing", "ensemble", "calibration", "launch-list",
                             "late-step"],
                    help="column: the 4M-particle granular column (default); footing: the "
                         "16M-particle footing on a slope over a foundation; ensemble: 512 "
                         "independent 2D slopes in one solver; calibration: derivatives of "
                         "the 256k-particle column's final positions with respect to (E, phi); "
                         "launch-list: one launch of every kernel (mixed and FP64 steps of a "
                         "1M-particle column, state conversions, records, one reversed "
                         "calibration step) inside a profiler start/stop window, for "
                         "ncu --profile-from-start off; late-step: the 1M-particle column "
                         "advanced --late-steps steps, then one step inside a profiler window "
                         "(prints no bench line)")
    ap.add_argument("--late-steps", type=int, default=2000,
                    help="late-step workload: steps before the profiled step")
    ap.add_argument("--profile-steps", type=int, default=20,
                    help="steps timed per kernel after the timed window")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-fp64-arm", action="store_true",
                    help="skip the FP64 run reported beside the mixed one")
    ap.add_argument("--launch-shape", default="",
                    help="p2g_tile,node_threads,return_blocks_per_sm to use instead of "
                         "autotuning (e.g. 128,256,8)")
    ap.add_argument("--autotune-steps", type=int, default=5,
                    help="steps per launch-shape candidate of the autotuner before the "
                         "warm-up (0 keeps the default launch shape)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    ap.add_argument("--accuracy-steps", default="50,500,2000",
                    help="steps at which the mixed path's deviation from the FP64 path (and "
                         "the FP64 path's own one-ulp floor) is reported; the last one also "
                         "starts the late timed window ('' skips both)")
    return ap.parse_args()


def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.barrier()
        torch.cuda.synchronize()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """Sample the SM clock and the clock-event (throttle) reasons of the
    bench's GPU during the timed region.

    A thread polls NVML as fast as it answers (a sample every few tens of
    microseconds): the timed region of a default run lasts tens of
    milliseconds, shorter than nvidia-smi's sampling period.  The step calls
    release the GIL, so the thread samples while the steps run.  The GPU is
    found by its UUID, so CUDA_VISIBLE_DEVICES does not matter."""
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, device):
        import threading
        self.samples = []  # (perf_counter, sm MHz, max sm MHz, reasons bitmask)
        self.window = [None, None]
        self.nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(device).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self.nvml, self.h = pynvml, h
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nvml = None
            return
        self.run = True
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()

    def _poll(self):
        nv, h = self.nvml, self.h
        while self.run:
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
            except Exception:
                break
            self.samples.append((time.perf_counter(), mhz, self.max_mhz, rs))
            if self.window[0] is None:
                time.sleep(0.002)  # before the timed region: sample slowly

    def mark_start(self):
        self.window[0] = time.perf_counter()

    def mark_end(self):
        self.window[1] = time.perf_counter()

    def stop(self):
        if self.nvml is None:
            return None
        self.run = False
        self.t.join(5)
        lo, hi = self.window
        rows = [r for r in self.samples if lo is not None and hi is not None and lo <= r[0] <= hi]
        in_window = bool(rows)
        if not rows:
            rows = self.samples[-3:]
        if not rows:
            return None
        reasons = sorted({n for *_, rs in rows for n, bit in self.REASONS if rs & bit})
        return {"sm_mhz": statistics.median(r[1] for r in rows),
                "sm_max_mhz": max(r[2] for r in rows), "reasons": reasons,
                "samples": len(rows), "in_timed_window": in_window, "source": "nvml"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def cpu_sample_problem():
    """A bounded sample of the workload for the CPU oracle: the same column at
    1/8 of its x-y footprint (mesh 50x25x50 cells, block 25x25x50 cells,
    250,000 particles), same material, boundary conditions and step."""
    from mpm_b200 import problems as P
    return P.column_3d(shape=(50, 25, 50), block=(25, 25, 50))


def time_cpu_oracle(seconds, warmup=1, max_steps=200):
    """particle-steps/s of the CPU oracle (all host threads) on the sample."""
    from oracle.oracle import build_oracle
    prob = cpu_sample_problem()
    threads = os.cpu_count() or 1
    o = build_oracle(prob, nthreads=threads)
    o.step(warmup)
    steps, t0 = 0, time.perf_counter()
    while steps < max_steps:
        o.step(1)
        steps += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    rate = prob.nparticles * steps / dt
    sample = (f"3D MohrCoulomb USL column, mesh 50x25x50 hex8, {prob.nparticles} particles "
              f"(1/8 of the 4M footprint), {steps} steps after {warmup} warm-up, "
              f"{dt:.1f} s wall, OpenMP {threads} threads")
    return rate, threads, sample


def run_reference(args, rank, world):
    """--impl reference: the reference CPU path (oracle port, the reference
    cannot be built here) on the box's host cores."""
    if rank != 0:
        return
    from oracle.oracle import build_oracle
    prob = cpu_sample_problem()
    threads = os.cpu_count() or 1
    o = build_oracle(prob, nthreads=threads)
    o.step(max(args.warmup, 1))
    t0 = time.perf_counter()
    o.step(args.steps)
    dt = time.perf_counter() - t0
    rate = prob.nparticles * args.steps / dt
    sample = (f"3D MohrCoulomb USL column, mesh 50x25x50 hex8, {prob.nparticles} particles, "
              f"{args.steps} steps, OpenMP {threads} threads")
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": rate,
        "unit": "particle-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "3D granular column collapse, MohrCoulomb USL FP64 (sample)"},
        "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def time_arm(prob, precision, args, world, dev, clocks=None):
    """Build a solver, run the warm-up, time K steps on the device (the
    production path: steps replayed from the captured CUDA graph), then time
    a short window per kernel (profiling launches eagerly)."""
    from mpm_b200 import problems as P
    t0 = time.perf_counter()
    s = P.build_solver(prob, precision=precision, device=dev)
    setup_s = time.perf_counter() - t0
    # launch shape timed on this state, then the state restored (or given)
    s.tune_report = None
    if args.launch_shape:
        s.set_launch_shape(*(int(v) for v in args.launch_shape.split(",")))
        s.tune_report = {"given": list(s.launch_shape())}
    elif args.autotune_steps:
        s.tune_report = s.autotune(args.autotune_steps)
    s.step(args.warmup)
    barrier(world)
    launches0 = s.launch_count
    if clocks:
        clocks.mark_start()
    ms = s.step_timed(args.steps)
    if clocks:
        clocks.mark_end()
    launches = s.launch_count - launches0
    ms = max_over_ranks(ms, world)
    s.set_profiling(True)
    s.step_timed(args.profile_steps)
    prof = s.kernel_profile()
    s.set_profiling(False)
    return s, ms, prof, launches, setup_s


def time_persistent(prob, args, world, dev):
    """The persistent form of the mixed USL step (every pass of K steps in one
    cooperative launch, grid barriers between the passes) timed like the
    per-pass graph arm: same warm-up, K steps per launch, device events; its
    results are bitwise those of the graph arm (tests/test_gpu_persistent.py)."""
    from mpm_b200 import problems as P
    s = P.build_solver(prob, precision="mixed", device=dev)
    s.set_persistent(args.steps)
    s.step(args.warmup)
    barrier(world)
    ms = max_over_ranks(s.step_timed(args.steps), world)
    n = s.nparticles
    s.step(2 * args.steps)  # untimed: a second full launch of a call replays the captured graph
    graph = s.persistent()[1]
    s.close()
    return {"ms_per_step": ms / args.steps, "value": world * n * args.steps / (ms / 1e3),
            "steps_per_launch": args.steps, "launches": 1, "graph_replayed_after_first": graph}


def field_errors(a, b):
    """max |a - b| / max |b| per field (F compared as F - I)."""
    out = {}
    for k in FIELDS:
        x, y = np.asarray(a[k], float), np.asarray(b[k], float)
        if k == "F":
            x, y = x - np.eye(3).reshape(1, 9), y - np.eye(3).reshape(1, 9)
        out[k] = float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))
    return out


def l2_errors(a, b):
    """||a - b||_2 / ||b||_2 over all particles and components, per field (F
    compared as F - I)."""
    out = {}
    for k in FIELDS:
        x, y = np.asarray(a[k], float), np.asarray(b[k], float)
        if k == "F":
            x, y = x - np.eye(3).reshape(1, 9), y - np.eye(3).reshape(1, 9)
        out[k] = float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    return out


def accuracy_and_late_window(prob, args, world, dev, checkpoints):
    """Mixed against FP64 at each checkpoint, beside the floor: FP64 against
    FP64 started from the initial stress moved by one ulp (the run's own
    conditioning).  Both max-norm (max |a-b| / max |b|) and L2 errors.  Then
    a late timed window of K steps on each path, after the last checkpoint."""
    from mpm_b200 import problems as P
    mixed = P.build_solver(prob, precision="mixed", device=dev)
    fp64 = P.build_solver(prob, precision="fp64", device=dev)
    pert = P.build_solver(prob, precision="fp64", device=dev)
    st = pert.read()
    st["stress"] = np.where(st["stress"] == 0.0, 0.0, np.nextafter(st["stress"], np.inf))
    pert.load(st)
    rows, done = [], 0
    for c in checkpoints:
        for s in (mixed, fp64, pert):
            s.step(c - done)
        done = c
        m, f, q = mixed.read(), fp64.read(), pert.read()
        rows.append({"step": c, "mixed_vs_fp64_max": field_errors(m, f),
                     "mixed_vs_fp64_l2": l2_errors(m, f),
                     "fp64_one_ulp_floor_max": field_errors(q, f),
                     "fp64_one_ulp_floor_l2": l2_errors(q, f)})
    del pert
    # the launch shape re-timed on the late state (the state is restored)
    tune_m = tune_f = None
    if args.launch_shape:
        for s in (mixed, fp64):
            s.set_launch_shape(*(int(v) for v in args.launch_shape.split(",")))
    elif args.autotune_steps:
        tune_m, tune_f = mixed.autotune(args.autotune_steps), fp64.autotune(args.autotune_steps)
    barrier(world)
    ms_m = max_over_ranks(mixed.step_timed(args.steps), world)
    ms_f = max_over_ranks(fp64.step_timed(args.steps), world)
    n = mixed.nparticles

    def kernels(s):
        s.set_profiling(True)
        s.step_timed(args.profile_steps)
        prof = s.kernel_profile()
        s.set_profiling(False)
        return {k: v[0] / v[1] for k, v in prof.items() if v[1]}
    late = {"after_step": done, "steps": args.steps,
            "value": world * n * args.steps / (ms_m / 1e3), "ms_per_step": ms_m / args.steps,
            "kernels_ms_per_launch": kernels(mixed), "launch_shape": tune_m,
            "fp64": {"value": world * n * args.steps / (ms_f / 1e3),
                     "ms_per_step": ms_f / args.steps, "kernels_ms_per_launch": kernels(fp64),
                     "launch_shape": tune_f}}
    return rows, late


def run_calibration(args, rank, world):
    """Config D: the FP64 forward run and the run carrying derivatives with
    respect to (E, phi), timed on the device, and the gradient of the loss
    |x_final - x_target|^2 (target run at E = 8e6, phi = 32) against central
    differences of the FP64 path (relative step 1e-6)."""
    from mpm_b200 import problems as P
    from mpm_b200.sensitivity import run_with_sensitivities
    params = [(0, "youngs_modulus"), (0, "friction")]
    theta = np.array([1e7, 30.0])
    dev = int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else 0
    build = lambda th: P.build_solver(P.config_d(phi=th[1], E=th[0]), precision="fp64", device=dev)

    def final_x(th):
        s = build(th)
        s.step(args.steps)
        x = s.read()["x"]
        s.close()
        return x

    def kernels(s):  # per-kernel ms per step over a 20-step eager window
        s.set_profiling(True)
        s.step_timed(20)
        prof = {k: round(v[0] / 20, 4) for k, v in s.kernel_profile().items() if v[1]}
        s.set_profiling(False)
        return prof

    f = build(theta)
    f.step(args.warmup)
    ms_f = max_over_ranks(f.step_timed(args.steps), world)
    n = f.nparticles
    fwd_kernels = kernels(f)
    f.close()
    t = build(theta)
    t.set_sensitivities(params)
    t.step(args.warmup)
    ms_t = max_over_ranks(t.step_timed(args.steps), world)
    tan_kernels = kernels(t)
    t.close()
    # the reverse sweep: record + reverse, on the host clock (both calls return
    # after their device work has finished); every step's start state kept
    # (no recompute), and checkpoints sqrt(steps) apart (least memory, every
    # segment recomputed)
    # as in a calibration loop: the first record allocates the tape, later
    # ones reuse it; each timed sweep starts from the same warmed-up state
    every_sqrt = int(np.ceil(np.sqrt(args.steps)))
    adj_times, adj_first = {}, {}
    for every in (1, every_sqrt):
        a = build(theta)
        a.step(args.warmup)
        st0 = a.read()
        ones = np.ones((a.nparticles, 3))
        for rep in range(2):
            a.load(st0)
            a.set_current_step(args.warmup)
            t0 = time.perf_counter()
            a.adjoint_record(args.steps, params, checkpoint_every=every)
            a.adjoint_reverse(dL_dx=ones)
            (adj_first if rep == 0 else adj_times)[every] = max_over_ranks(
                time.perf_counter() - t0, world)
        a.close()
    adj_s = adj_times[1]
    # the same again with per-kernel events (eager launches)
    a = build(theta)
    a.step(args.warmup)
    a.set_profiling(True)
    a.adjoint_record(args.steps, params, checkpoint_every=1)
    a.adjoint_reverse(dL_dx=ones)
    adj_kernels = {k: {"total_ms": v[0], "launches": v[1]} for k, v in a.kernel_profile().items()
                   if v[1]}
    a.set_profiling(False)
    a.close()
    target = final_x((8e6, 32.0))
    x, J = run_with_sensitivities(build, theta, params, args.steps)
    grad = 2.0 * np.einsum("pd,kpd->k", x - target, J)
    s_adj = build(theta)
    _, grad_adj = s_adj.adjoint_run(args.steps, params, target, checkpoint_every=every_sqrt)
    s_adj.close()
    fd = []
    for k in range(2):
        h = 1e-6 * theta[k]
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd.append((np.sum((final_x(tp) - target) ** 2) - np.sum((final_x(tm) - target) ** 2))
                  / (2 * h))
    if rank == 0:
        value = world * n * args.steps / (ms_t / 1e3)
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_t / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 + 2 tangents", "data": "synthetic",
            "config": {"workload": f"calibration column (config D): 80x40x30 hex8 dx=0.02, {n} "
                                   f"particles, MohrCoulomb c=1 kPa, USL, dt=1e-5, derivatives "
                                   f"w.r.t. (E, phi)", "particles": n},
            "forward": {"value": world * n * args.steps / (ms_f / 1e3),
                        "ms_per_step": ms_f / args.steps},
            "tangent_over_forward": ms_t / ms_f,
            "kernels_ms_per_step": {"forward": fwd_kernels, "tangent": tan_kernels},
            "adjoint": {"seconds": adj_s, "checkpoint_every": 1,
                        "over_forward": adj_s / (ms_f / 1e3), "kernels": adj_kernels,
                        "first_call_seconds": adj_first[1],
                        "sqrt_checkpoints": {"checkpoint_every": every_sqrt,
                                             "seconds": adj_times[every_sqrt],
                                             "first_call_seconds": adj_first[every_sqrt],
                                             "over_forward": adj_times[every_sqrt] / (ms_f / 1e3)},
                        "note": "record (forward keeping checkpoints) + reverse sweep (segment "
                                "recompute + reverse kernels), host clock around both, against "
                                "the device time of the plain forward run; seconds: a repeated "
                                "sweep (the tape's buffers kept), first_call_seconds: the first, "
                                "which allocates them; the gradient below comes from the "
                                "sqrt-spaced checkpoints"},
            "gradient": {"loss": "sum |x_final - x_target|^2, target E=8e6, phi=32",
                         "at": theta.tolist(), "tangent": grad.tolist(),
                         "adjoint": [float(v) for v in grad_adj], "central_fd": fd,
                         "fd_relative_step": 1e-6,
                         "relative_error": [abs(g - d) / max(abs(d), 1e-300)
                                            for g, d in zip(grad, fd)]},
        }
        print(json.dumps(line), flush=True)


def run_late_step(args):
    """The 1M-particle column advanced --late-steps steps (most points plastic
    by step 2000), its per-kernel times over 5 profiled steps, then one step
    inside a profiler window (for ncu --profile-from-start off)."""
    import torch
    from mpm_b200 import problems as P
    s = P.build_solver(P.column_3d(block=(50, 50, 50)), precision=args.precision)
    s.step(args.late_steps)
    ys = s.read()["svars"][:, 0]
    s.set_profiling(True)
    s.step_timed(5)
    prof = {k: round(v[0] / v[1], 4) for k, v in s.kernel_profile().items() if v[1]}
    s.set_profiling(False)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    s.step(1)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"workload": "late-step", "precision": args.precision,
                      "after_step": args.late_steps, "particles": s.nparticles,
                      "plastic_fraction": float(np.mean(ys != 0)), "kernels_ms_per_launch": prof}))


def run_launch_list():
    """One launch of every kernel of the product inside a profiler window
    (cudaProfilerStart/Stop), for a launch list with per-kernel DRAM bytes:
    a mixed and an FP64 step of the 1M-particle column (eager launches), the
    host-row/device-layout conversions both ways, the PODParticle records, a
    slab step's halo pack / unpack and layer count, one step of the
    calibration column carrying derivatives, one recorded and reversed step of
    it, and the batch constitutive update of 262,144 MohrCoulomb points."""
    import torch
    from mpm_b200 import problems as P
    from mpm_b200.solver import material_stress_batch
    col = P.column_3d(block=(50, 50, 50))
    m = P.build_solver(col, precision="mixed")
    m.step(5)
    m.set_profiling(True)
    f = P.build_solver(col, precision="fp64")
    f.step(5)
    f.set_profiling(True)
    cal = P.build_solver(P.config_d(), precision="fp64")
    cal.step(3)
    tan = P.build_solver(P.config_d(), precision="fp64")
    tan.step(3)
    tan.set_sensitivities([(0, "youngs_modulus"), (0, "friction")])
    st = m.read()
    n = cal.nparticles
    halo = torch.empty(f.halo_bytes(), dtype=torch.uint8, device="cuda")
    props = P.mohr_coulomb(1e7, 0.3, 1800., 30., 1000., 0.)
    rng = np.random.default_rng(7)
    npts = 1 << 18
    sig = np.tile(np.array([-2e4, -2e4, -4e4, 0., 0., 0.]), (npts, 1)) * rng.uniform(0.5, 1.5, (npts, 1))
    deps = rng.normal(0.0, 2e-4, (npts, 6))
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    m.step(1)
    f.step(1)
    m.load(st)
    m.read()
    f.write_pod()
    f.step_begin()
    f.halo_pack(10, halo.data_ptr())
    f.halo_unpack(10, halo.data_ptr())
    f.step_end()
    f.layer_count(10, 190)
    tan.step(1)
    cal.adjoint_record(1, [(0, "youngs_modulus"), (0, "friction")], checkpoint_every=1)
    cal.adjoint_reverse(dL_dx=np.ones((n, 3)))
    material_stress_batch(3, "MohrCoulomb3D", props, sig, deps, 1800.)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"workload": "launch-list", "particles": [m.nparticles, n]}))


def main():
    args = parse()
    rank, world = dist_init(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "calibration":
        run_calibration(args, rank, world)
        return
    if args.workload == "launch-list":
        run_launch_list()
        return
    if args.workload == "late-step":
        run_late_step(args)
        return
    from mpm_b200 import problems as P
    block = tuple(int(v) for v in args.block.split(","))
    if args.workload == "column":
        prob = P.config_b(block=block)
    elif args.workload == "footing":
        prob = P.config_e()
    else:
        from mpm_b200 import ensemble as E
        prob, _ = E.ensemble_problem(E.random_runs(512))
    dev = int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else 0
    clocks = Clocks(dev)
    s, ms, prof, launches, setup_s = time_arm(prob, args.precision, args, world, dev, clocks)
    clk = clocks.stop()
    n = s.nparticles
    value = world * n * args.steps / (ms / 1e3)
    state = s.read()

    # the FP64 path on the same workload and steps, with the mixed path's
    # per-field deviation from it
    fp64 = None
    if args.precision == "mixed" and not args.no_fp64_arm:
        s64, ms64, prof64, _, _ = time_arm(prob, "fp64", args, world, dev)
        fp64 = {"value": world * n * args.steps / (ms64 / 1e3), "ms_per_step": ms64 / args.steps,
                "kernels_ms_per_launch": {k: v[0] / v[1] for k, v in prof64.items() if v[1]},
                "mixed_vs_fp64_field_errors": field_errors(state, s64.read())}
        del s64

    # the persistent form of the same step (one launch for the K steps)
    persistent = None
    if args.precision == "mixed" and prob.analysis.get("scheme", "usl") == "usl":
        persistent = time_persistent(prob, args, world, dev)
        persistent["graph_over_persistent"] = (ms / args.steps) / persistent["ms_per_step"]

    # end to end through the public API with the state in page-locked host
    # arrays (the library's pinned_empty; pageable arrays if the host cannot
    # pin them): load, K steps, read back into host arrays
    from mpm_b200 import MPMError
    try:
        st, outb, host_mem = s.state_buffers(pinned=True), s.state_buffers(pinned=True), "page-locked"
    except MPMError:
        st, outb, host_mem = s.state_buffers(), s.state_buffers(), "pageable"
    for k in st:
        if k in ("x", "u", "v"):
            st[k][:] = 0.0
            st[k][:, :prob.dim] = state[k]
        else:
            st[k][...] = state[k]
    h2d = sum(np.asarray(st[k]).nbytes for k in st)
    barrier(world)
    t1 = time.perf_counter()
    s.load(st)
    s.step(args.steps)
    out = s.read(out=outb)
    e2e_s = max_over_ranks(time.perf_counter() - t1, world)
    d2h = sum(np.asarray(outb[k]).nbytes for k in outb)
    e2e = {"value": world * n * args.steps / e2e_s, "unit": "particle-steps/s",
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
           "host_memory": host_mem}
    del out

    # roofline of the dominant kernel
    peak, peak_kind = measured_peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    name, (tot_ms, cnt) = dom
    avg_s = tot_ms / max(cnt, 1) / 1e3
    bpp = BYTES_PER_PARTICLE[(args.precision, prob.dim)]
    bytes_launch = bpp.get(name, 0) * n
    achieved = bytes_launch / avg_s / 1e9
    total = max(sum(x[0] for x in prof.values()), 1e-30)
    roofline = {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "bytes_per_particle": bpp.get(name, 0), "bytes_per_launch": bytes_launch,
                "avg_launch_ms": avg_s * 1e3,
                "traffic": (MEASURED_TRAFFIC_PER_PARTICLE.get((args.precision, prob.dim), {})
                            .get(name, 0.0) * n) or None,
                "traffic_source": "ncu dram bytes per particle on the 1M-particle column, "
                                  "scaled to this launch's particles",
                "kernel_shares": {k: v[0] / total for k, v in prof.items() if v[1]}}

    # whole-step roofline (bytes per particle-step of the step, not of one kernel)
    sbytes = STEP_BYTES_PER_PARTICLE[(args.precision, prob.dim)]
    roofline["step"] = {"bytes_per_particle_step": sbytes,
                        "achieved": value / world * sbytes / 1e9, "unit": "GB/s",
                        "frac": value / world * sbytes / 1e9 / peak}

    accuracy, late = None, None
    checkpoints = [int(v) for v in args.accuracy_steps.split(",") if v.strip()]
    if checkpoints and args.precision == "mixed" and not args.no_fp64_arm:
        accuracy, late = accuracy_and_late_window(prob, args, world, dev, checkpoints)
        late["roofline_step_frac"] = late["value"] / world * sbytes / 1e9 / peak

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "column":
        rate, threads, sample = time_cpu_oracle(args.cpu_sample_seconds)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": threads, "kind": "port",
               "sample": sample}

    if rank == 0:
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPES[args.precision], "data": "synthetic",
            "config": {"workload": (f"3D granular column collapse, MohrCoulomb USL FLIP "
                                    f"{args.precision.upper()}, 200x100x50 hex8 dx=0.01, "
                                    f"{n} particles") if args.workload == "column" else
                                   (f"3D footing on a MohrCoulomb slope over a LinearElastic "
                                    f"foundation, USL FLIP {args.precision.upper()}, 400x200x100 "
                                    f"hex8 dx=0.005, {n} particles") if args.workload == "footing"
                                   else (f"512 independent 2D MohrCoulomb slopes in one solver "
                                         f"(N ~ U[2000, 40000], phi ~ U[20, 40], c ~ U[0, 5 kPa]), "
                                         f"USL FLIP {args.precision.upper()}, dx=0.01, {n} "
                                         f"particles"),
                       "particles": n, "nodes": prob.nnodes, "cells": prob.ncells,
                       "dt": prob.analysis["dt"], "precision": args.precision,
                       "l2": "state larger than L2 (no flush needed)",
                       "kernel_profile_steps": args.profile_steps,
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "setup_s": setup_s},
            "fp64": fp64, "persistent": persistent,
            "accuracy": accuracy, "late": late,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk, "launch_shape": s.tune_report,
            "kernels": {k: {"total_ms": v[0], "launches": v[1]}
                                       for k, v in prof.items() if v[1]},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
