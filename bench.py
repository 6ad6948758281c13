"""Benchmark of the single-partition MLS-MPM step (particle-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload block8m] [--precision mixed|fp64]

Workload: the 8,000,000-particle block of the mixed-precision target
configuration (4.0 x 1.0 x 1.0 m, h = 0.01 m, dt = 5e-6 s, lognormal cohesion
median 3e5 Pa sigma_log 0.3, indenter 1.0 m/s), seeded synthetic jittered
lattice. One "step" is one substep of Model3D::Step on the whole block.

value: particle-steps/s over all ranks with the state resident on the device
(timed with CUDA events on the handle's stream, barrier + synchronize on both
sides, max over ranks). e2e: the same metric through the public C-ABI with
host buffers (pinned SoA and cohesion uploaded, the cell-key sort, K substeps
with the force history read back, SoA downloaded) inside the timed region. N > 1 runs independent
replicas, one per GPU (the path is one partition; no collective).

--io times the IO around the step (frame records, snapshot write/read,
download/upload).

--partitions N times N x-slab partitions (the in-process driver) against
one partition of the same driver on the same block (--halo slabs).

--impl reference times the reference's own step kernels (mpm_kernels.cuh
compiled as host C++ from its source into oracle/_ref, OpenMP on all host
cores; the oracle port when that build is absent), without loading the
product library: exactly K substeps, each over a bounded sample of the same
workload (a shorter block of the same cross-section, h, density, material
and indenter, sized so that the run takes about --ref-seconds).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

B_PARTICLE = {"mixed": 208, "fp64": 416}       # bytes per particle-step (state read + write)
B_COHESION = {"mixed": 4, "fp64": 8}           # per-particle cohesion read
B_NODE = {"mixed": 32, "fp64": 64}             # bytes per active node per step


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="block8m")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--accum", default="float", choices=["float", "fixed"],
                    help="mixed P2G grid accumulation: FP32 float4 atomics or 64-bit fixed point")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-arm", action="store_true", help="skip the plain FP64 step on the same block")
    ap.add_argument("--fp64-steps", type=int, default=300, help="substeps of the FP64 arm (at most --steps)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=45.0,
                    help="target length of the reference arm's timed part (sizes its per-substep sample)")
    ap.add_argument("--adjoint", action="store_true",
                    help="time the adjoint (forward with checkpoints + reverse sweep) on the calibration workload")
    ap.add_argument("--ckpt-every", type=int, default=20)
    ap.add_argument("--partitions", type=int, default=0,
                    help="time N x-slab partitions in this process (mpm_multi_*, on --gpus devices) "
                         "against one partition of the same driver on the same block")
    ap.add_argument("--io", action="store_true",
                    help="time the IO around the step: animation-frame records, SoA download, snapshot "
                         "write and read, upload")
    ap.add_argument("--halo", type=int, default=15,
                    help="GridHaloSize of the --partitions run (the reference's default is 15)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world, backend):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, value, device):
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms; stop()
    keeps the samples that arrived inside the timed window [t0, t1]."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self, t0=None, t1=None):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for t, ln in self.lines:
            if t0 is not None and not (t0 <= t <= t1):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_particle(kernel):
    """DRAM bytes per particle of the dominant kernel from the committed ncu
    summary profiles/<kernel>_<workload>.md (line `dram_bytes_per_particle:`),
    captured on a smaller block and scaled by particles."""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", f"{kernel}_*.md"))):
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_particle:"):
                    return float(line.split(":", 1)[1].split()[0])
    return None


def reference_cpu(threads):
    """The reference step on the host cores, without the product library:
    (make(cfg) -> (sim, n), kind, what). With oracle/_ref/libref_mpm.so (the
    reference's own mpm_kernels.cuh compiled as host C++ from its source) the
    sim is oracle.pyoracle.RefSim, kind "reference"; without it, the oracle
    port (kind "port"). The parameter blocks come from the oracle's own
    restatement of SimParams3D's routines. The reference kernels have no
    per-particle cohesion: RefSim runs the workload's median cohesion through
    the global DP_threshold_p (the same work per particle). The input is
    sorted by cell key first, as the reference's RemoveDisabledAndSort does
    after loading."""
    from icempm_3dm_b200 import generator as gen
    from oracle import params as oracle_params
    from oracle import pyoracle as po
    use_ref = po.ref_mpm_lib() is not None

    def make(c):
        prms, soa, coh = gen.make_block(c, ops=oracle_params.OPS)
        n = soa.shape[1]
        perm = po.sort_permutation(prms, soa, n)
        soa = np.ascontiguousarray(soa[:, perm])
        if use_ref:
            return po.RefSim(prms, soa, n, nthreads=threads), n
        p0 = None if coh is None else coh[perm] / prms.DP_tan_phi
        return po.OracleSim(prms, soa, n, p0=p0, svd_mode=0, nthreads=threads), n

    if use_ref:
        what = (f"the reference's own mpm_kernels.cuh compiled as host C++ (oracle/_ref/libref_mpm.so), "
                f"FP64 with its FP32 SVD, OpenMP {threads} threads, median cohesion")
        return make, "reference", what
    return make, "port", f"oracle port of the reference step, FP64, OpenMP {threads} threads"


def cpu_baseline(cfg_name, seconds, threads=None):
    """The reference step on the host cores (reference_cpu) on the same
    block: warm-up 1 substep, then substeps until `seconds` have elapsed (at
    least 2)."""
    from icempm_3dm_b200 import generator as gen
    threads = threads or os.cpu_count() or 1
    make, kind, what = reference_cpu(threads)
    sim, n = make(gen.CONFIGS[cfg_name])
    sim.step(1)
    t0 = time.perf_counter()
    done = 0
    while done < 2 or time.perf_counter() - t0 < seconds:
        sim.step(1)
        done += 1
    dt = time.perf_counter() - t0
    return {"value": n * done / dt, "unit": "particle-steps/s", "cores": threads, "kind": kind,
            "sample": f"{done} substeps of the full {n}-particle block after 1 warm-up substep ({what})"}


def reference_sample(cfg, n_s):
    """A bounded sample of a block workload: the same cross-section, h, dt,
    particle density, material, cohesion law and indenter, with the block's
    length in x (and the grain count of a grains workload) scaled by n_s / n,
    so the grid shrinks with the particle count."""
    import dataclasses
    f = n_s / cfg.n
    dims = (cfg.dims[0] * f, cfg.dims[1], cfg.dims[2])
    kw = {"grains": max(1, round(cfg.grains * f))} if cfg.grains else {}
    return dataclasses.replace(cfg, name=cfg.name + "_sample", n=n_s, dims=dims, **kw)


def run_reference(args):
    """The reference step on all host cores (reference_cpu; the product
    library is not loaded): exactly --steps substeps, each over a bounded
    sample of the workload sized from one probe substep of the full block so
    that the timed part takes about --ref-seconds (the full block when that
    fits)."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from icempm_3dm_b200 import generator as gen
    threads = os.cpu_count() or 1
    cfg = gen.CONFIGS[args.workload]
    make, kind, what = reference_cpu(threads)
    sim, n_full = make(cfg)
    t0 = time.perf_counter()
    sim.step(1)
    rate = n_full / (time.perf_counter() - t0)        # probe: particle-substeps/s on this host
    n_s = min(n_full, max(20_000, int(rate * args.ref_seconds / max(args.steps, 1))))
    if n_s < n_full:
        scfg = reference_sample(cfg, n_s)
        sim, n = make(scfg)
        sample = (f"{n} particles per substep: a {scfg.dims[0]:.3f} x {scfg.dims[1]:g} x {scfg.dims[2]:g} m block "
                  f"of the {cfg.name} workload (same h, dt, density, material, cohesion law, indenter)")
    else:
        n = n_full
        sample = f"the full {n}-particle {cfg.name} block"
    sim.step(max(1, min(args.warmup, 3)))
    t0 = time.perf_counter()
    hist, err = sim.step(args.steps)
    dt = time.perf_counter() - t0
    if err:
        print(f"reference step reported error code {err}", file=sys.stderr)
    value = n * args.steps / dt
    out = {"impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
           "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": {"workload": args.workload, "particles": n_full},
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": threads, "kind": kind,
                            "sample": f"{args.steps} substeps of {sample} ({what})"},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def fp64_arm(args, prms, soa, coh, local, stream, dist, world):
    """The plain FP64 step (FP64 state and transfers, the reference's FP32
    SVD) on the same block in the same process: min(--steps, --fp64-steps)
    substeps after 3 warm-up substeps, CUDA events on the handle's stream, max
    over ranks; its dominant kernel's roofline from the in-library per-kernel
    events."""
    import torch
    from icempm_3dm_b200 import MPMHandle, PRECISION_FP64
    n = soa.shape[1]
    steps = max(1, min(args.steps, args.fp64_steps))
    device = torch.device("cuda", local)
    h = MPMHandle(prms, n, PRECISION_FP64, device=local)
    try:
        h.set_stream(stream.cuda_stream)
        h.upload(soa, cohesion=coh)
        h.sort()
        h.step(3, want_forces=False)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h.step(steps)
        e1.record(stream)
        e1.synchronize()
        ms = max_over_ranks(dist, e0.elapsed_time(e1), device)
        kms = h.step_timed(steps)
        active = h.active_nodes()
    finally:
        h.close()
    names = ["grid clear", "k_p2g_pairs_f64", "k_update_f64", "k_g2p_f64"]
    k = int(np.argmax(kms[1:])) + 1
    dom_ms = kms[k] / steps
    # FP64 form: P2G reads 200 B (utility, x, v, F, C) and writes the grid
    # (32 B per active node); G2P reads 112 B (+ 8 B cohesion) and the grid
    # (32 B per node), writes 208 B
    per = {1: 200, 3: 320 + (8 if coh is not None else 0)}.get(k, 0)
    dom_bytes = n * per + active * 32
    peak, peak_kind = measured_peak_hbm()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    step_bytes = n * (B_PARTICLE["fp64"] + (B_COHESION["fp64"] if coh is not None else 0)) + active * B_NODE["fp64"]
    return {"value": world * n * steps / (ms * 1e-3), "unit": "particle-steps/s", "steps": steps,
            "ms_per_step": ms / steps, "dtype": "f64",
            "kernel_ms_per_step": {"clear": kms[0] / steps, "p2g": kms[1] / steps, "update": kms[2] / steps,
                                   "g2p": kms[3] / steps},
            "hbm_fraction_step": step_bytes / (ms / steps * 1e-3) / 1e9 / peak,
            "roofline": {"bound": "hbm", "kernel": names[k], "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak}}


def run_ours(args):
    import torch
    world, rank, local = dist_env()
    if world != args.gpus and world > 1:
        print(f"warning: WORLD_SIZE {world} != --gpus {args.gpus}", file=sys.stderr)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = init_dist(world, "nccl")

    from icempm_3dm_b200 import MPMHandle, PRECISION_FP64, PRECISION_MIXED
    from icempm_3dm_b200 import generator as gen
    prec = PRECISION_MIXED if args.precision == "mixed" else PRECISION_FP64
    cfg = gen.CONFIGS[args.workload]
    prms, soa, coh = gen.make_block(cfg)
    n = soa.shape[1]
    stream = torch.cuda.Stream(device=device)

    h = MPMHandle(prms, n, prec, device=local)
    h.set_stream(stream.cuda_stream)
    if args.accum == "fixed":
        h.set_grid_accumulation(1)
    h.upload(soa, cohesion=coh)
    h.sort()
    h.step(max(args.warmup, 3), want_forces=False)

    # --- device-resident throughput
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t_start = time.monotonic()
    e0.record(stream)
    hist = h.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    t_end = time.monotonic()
    torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop(t_start, t_end)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(dist, ms, device)
    value = world * n * args.steps / (ms_max * 1e-3)

    # --- per-kernel timing (CUDA events on the handle's stream, in-library)
    kms = h.step_timed(args.steps)
    active = h.active_nodes()
    if prec == PRECISION_MIXED:
        # the fused kernel carries the step's particle state and grid traffic;
        # the return map of crushed points runs in its own (small) kernel
        dom_name, dom_ms = "k_g2p2g_mixed", kms[3] / args.steps
        dom_bytes = n * (B_PARTICLE["mixed"] + (B_COHESION["mixed"] if coh is not None else 0)) + \
            active * B_NODE["mixed"]
        launches_per_step = 3
    else:
        names = ["grid clear", "k_p2g_pairs_f64", "k_update_f64", "k_g2p_f64"]
        k = int(np.argmax(kms[1:])) + 1
        dom_name, dom_ms = names[k], kms[k] / args.steps
        # FP64 form: P2G reads 200 B (utility, x, v, F, C), G2P reads 112 B
        # (+ 8 B cohesion) and writes 208 B
        per = {1: 200, 3: 320 + (8 if coh is not None else 0)}.get(k, 0)
        dom_bytes = n * per + (active * 32 if k in (1, 3) else active * 64)
        launches_per_step = 3
    peak, peak_kind = measured_peak_hbm()
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    tpp = traffic_per_particle(dom_name)
    step_bytes = n * (B_PARTICLE[args.precision] + (B_COHESION[args.precision] if coh is not None else 0)) + \
        active * B_NODE[args.precision]

    # --- end to end through the C-ABI with pinned host buffers
    host = torch.empty(soa.shape, dtype=torch.float64, pin_memory=True)
    host.numpy()[...] = soa
    host_np = host.numpy()
    out_host = torch.empty(soa.shape, dtype=torch.float64, pin_memory=True).numpy()
    h2 = MPMHandle(prms, n, prec, device=local)
    h2.set_stream(stream.cuda_stream)
    if args.accum == "fixed":
        h2.set_grid_accumulation(1)
    h2.upload(host_np, cohesion=coh)
    h2.sort()
    h2.step(3, want_forces=False)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    h2.upload(host_np, cohesion=coh)
    h2.sort()                    # cell order, as the reference's RemoveDisabledAndSort
    h2.step(args.steps)
    from icempm_3dm_b200._lib import LIB, dptr
    import ctypes
    nn = ctypes.c_uint(0)
    LIB.mpm_download_soa(h2._h, dptr(out_host), out_host.shape[1], ctypes.byref(nn))
    f1.record(stream)
    f1.synchronize()
    e2e_ms = max_over_ranks(dist, f0.elapsed_time(f1), device)
    h2.close()
    soa_bytes = soa.nbytes + (coh.nbytes if coh is not None else 0)
    e2e = {"value": world * n * args.steps / (e2e_ms * 1e-3), "unit": "particle-steps/s",
           "h2d_bytes_per_step": soa_bytes / args.steps,
           "d2h_bytes_per_step": (soa.nbytes + 24 * args.steps) / args.steps,
           "calls": "mpm_upload_soa + mpm_upload_cohesion + mpm_sort + mpm_step(K) + mpm_download_soa"}

    # --- the plain FP64 step on the same block (the "mixed vs FP64" ratio)
    fp64 = None
    if prec == PRECISION_MIXED and not args.no_fp64_arm:
        fp64 = fp64_arm(args, prms, soa, coh, local, stream, dist, world)

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(args.workload, args.cpu_seconds)

    if rank == 0:
        out = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if prec == PRECISION_MIXED else "f64",
            "data": "synthetic: seeded jittered-lattice ice block (shapes of the target configuration)",
            "config": {"workload": args.workload, "particles": n, "precision": args.precision,
                       "grid_accumulation": args.accum if prec == PRECISION_MIXED else "fp64",
                       "grid": [prms.GridXTotal, prms.GridY, prms.GridZ], "h": prms.cellsize,
                       "dt": prms.InitialTimeStep, "parallelism": f"replicas x{world}",
                       "l2": "state larger than L2 (no flush needed)",
                       "active_nodes": active, "step_bytes_algorithmic": step_bytes,
                       "hbm_fraction_step": step_bytes / (ms_max / args.steps * 1e-3) / 1e9 / peak},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": (tpp * n if tpp else None)},
            "kernel_ms_per_step": ({"update": kms[2] / args.steps, "g2p2g": kms[3] / args.steps,
                                    "return_map": kms[1] / args.steps} if prec == PRECISION_MIXED else
                                   {"update": kms[2] / args.steps, "g2p": kms[3] / args.steps,
                                    "p2g": kms[1] / args.steps, "clear": kms[0] / args.steps}),
            "force_last": hist[-1].tolist(),
            "fp64": fp64, "cpu_baseline": base, "e2e": e2e, "clocks": clocks,
            "gpu_launches": launches_per_step * args.steps,
        }
        print(json.dumps(out), flush=True)
    h.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_adjoint(args):
    """One JSON line: the adjoint (mpm_adjoint_forward with a checkpoint every
    --ckpt-every substeps, then mpm_adjoint_backward) on the calibration
    workload (default calib500k: 500,000 particles, 200 substeps), as
    particle-steps/s of forward + reverse together, beside the plain step of
    the same precision on the same block. --precision mixed (the default)
    runs the forward in mixed precision, with FP64 checkpoints and the FP64
    recompute in the reverse sweep; fp64 runs it in FP64 with the FP64 SVD.
    CUDA events on the handle's stream."""
    import torch
    from icempm_3dm_b200 import MPMHandle, PRECISION_FP64_SVD64, PRECISION_MIXED
    from icempm_3dm_b200 import generator as gen
    torch.cuda.set_device(0)
    cfg = gen.CONFIGS[args.workload if args.workload != "block8m" else "calib500k"]
    prms, soa, coh = gen.make_block(cfg)
    if coh is None:
        coh = cfg.cohesion_median * np.ones(soa.shape[1])
    n = soa.shape[1]
    steps = args.steps if args.steps != 1500 else cfg.steps
    stream = torch.cuda.Stream()
    prec = PRECISION_MIXED if args.precision == "mixed" else PRECISION_FP64_SVD64
    h = MPMHandle(prms, n, prec)
    h.set_stream(stream.cuda_stream)
    rng = np.random.default_rng(0)
    w = rng.standard_normal((steps, 3))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    h.upload(soa, cohesion=coh)
    h.step(max(args.warmup, 3))
    h.upload(soa, cohesion=coh)
    torch.cuda.synchronize()
    ev[0].record(stream)
    h.step(steps)
    ev[1].record(stream)
    # one untimed adjoint first: its checkpoint and grid buffers are allocated then
    h.upload(soa, cohesion=coh)
    h.adjoint_forward(steps, args.ckpt_every)
    h.adjoint_backward(w)
    h.upload(soa, cohesion=coh)
    torch.cuda.synchronize()
    ev[2].record(stream)
    h.adjoint_forward(steps, args.ckpt_every)
    h.adjoint_backward(w)
    ev[3].record(stream)
    ev[3].synchronize()
    t_fwd = ev[0].elapsed_time(ev[1])
    t_adj = ev[2].elapsed_time(ev[3])
    h.close()
    out = {"metric": "adjoint particle-steps/s (forward with checkpoints + reverse)",
           "value": n * steps / (t_adj * 1e-3), "unit": "particle-steps/s", "n_gpus": 1, "steps": steps,
           "higher_is_better": True, "dtype": "f64", "data": "synthetic",
           "config": {"workload": cfg.name, "particles": n, "ckpt_every": args.ckpt_every,
                      "forward_precision": args.precision},
           "ms_adjoint": t_adj, "ms_plain_forward": t_fwd, "adjoint_over_forward": t_adj / t_fwd}
    print(json.dumps(out), flush=True)
    return 0


def run_partitions(args):
    """One JSON line: the x-slab partitions of the reference's multi-partition
    GPU_Implementation6 (the in-process driver mpm_multi_*: halo exchange after
    every P2G, point transfers, the transfer-frequency rule and rebalance) with
    --partitions partitions, against the same driver with one partition, on
    the same block (GridHaloSize --halo). Partition i runs on device i % --gpus
    (not under torchrun: one process drives all devices). Wall clock around
    --steps substeps after --warmup; each call ends with the force history
    read back, so the clock covers all device work and the driver's own host
    time."""
    import dataclasses
    import torch
    from icempm_3dm_b200 import PRECISION_FP64, PRECISION_MIXED
    from icempm_3dm_b200 import generator as gen
    from icempm_3dm_b200.partitions import PartitionedSim
    prec = PRECISION_MIXED if args.precision == "mixed" else PRECISION_FP64
    cfg = dataclasses.replace(gen.CONFIGS[args.workload], halo=args.halo)
    prms, soa, coh = gen.make_block(cfg)
    n = soa.shape[1]
    devices = tuple(range(max(args.gpus, 1)))
    runs = {}
    for nparts in (1, args.partitions):
        p = prms.copy()
        p.nPartitions = nparts
        with PartitionedSim(p, n, prec, devices=devices) as m:
            m.upload(soa, cohesion=coh)
            m.step(max(args.warmup, 3))
            for d in devices:
                torch.cuda.synchronize(d)
            t0 = time.perf_counter()
            hist = m.step(args.steps)
            for d in devices:
                torch.cuda.synchronize(d)
            ms = (time.perf_counter() - t0) * 1e3
            most, rebalances, ptf = m.stats()
            moved = sum(nd for _, _, _, nd in m.info())
        runs[nparts] = {"value": n * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
                        "points_moved": moved, "largest_transfer": most, "rebalances": rebalances,
                        "point_transfer_frequency": ptf, "force_norm": float(np.linalg.norm(hist))}
    one, many = runs[1], runs[args.partitions]
    out = {"metric": "particle-steps/s", "value": many["value"], "unit": "particle-steps/s",
           "n_gpus": len(devices), "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": many["ms_per_step"], "higher_is_better": True, "scaling": "strong",
           "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
           "config": {"workload": args.workload, "particles": n, "precision": args.precision,
                      "partitions": args.partitions, "devices": list(devices), "halo": args.halo,
                      "timing": "wall clock around mpm_multi_step"},
           "one_partition": one, "partitioned": many,
           "partitioned_over_one": many["value"] / one["value"]}
    print(json.dumps(out), flush=True)
    return 0


def run_io(args):
    """One JSON line: the IO of the reference's SnapshotManager and
    transfer_from_device around the step, on the block after --warmup
    substeps, each by wall clock (seconds):
      - frame_full / frame_partial: mpm_frame_records, the records of a full
        animation frame (VisualPoint per point) and of a partial frame 1,000
        substeps later (UpdatePos / UpdateJp / UpdateStatus), built on the
        device and copied into preallocated host arrays;
      - save_frame_full / save_frame_partial: v%05d.h5 written by the HDF5
        codec (deflate 5, as the reference; chunks compressed on a thread
        pool);
      - download: mpm_download_soa of the 28-row FP64 SoA into a new array;
        download_pinned / upload_pinned: the same into and out of page-locked
        memory (pinned_empty, as the reference's HostSideSOA buffer);
      - save_snapshot / read_snapshot: d%05d.h5, uncompressed;
      - upload: mpm_upload_soa + mpm_upload_cohesion of the SoA read back.
    cpu_baseline: the float32 CPU restatement of the frame-record logic
    (oracle/frames.py, numpy) on the downloaded SoA, full and partial."""
    import ctypes
    import shutil
    import tempfile
    import torch
    from icempm_3dm_b200 import MPMHandle, PRECISION_FP64, PRECISION_MIXED, pinned_empty
    from icempm_3dm_b200 import generator as gen
    from icempm_3dm_b200 import snapshot as snap
    from icempm_3dm_b200._lib import LIB, check
    torch.cuda.set_device(0)
    prec = PRECISION_MIXED if args.precision == "mixed" else PRECISION_FP64
    cfg = gen.CONFIGS[args.workload]
    prms, soa, coh = gen.make_block(cfg)
    n = soa.shape[1]
    h = MPMHandle(prms, n, prec)
    h.upload(soa, cohesion=coh)
    h.sort()
    h.step(max(args.warmup, 3))
    t = {}

    def clock(name, fn):
        t0 = time.perf_counter()
        r = fn()
        t[name] = time.perf_counter() - t0
        return r

    pts = np.zeros(n, dtype=snap.VISUAL_POINT)
    pv, jp, st = (np.zeros(n, dtype=d) for d in (snap.UPDATE_POS, snap.UPDATE_JP, snap.UPDATE_STATUS))
    cnt = [ctypes.c_uint(0) for _ in range(4)]

    def full_records(frame):
        check(LIB.mpm_frame_records(h._h, frame, 1, pts.ctypes.data, ctypes.byref(cnt[0]), None, None, None, None,
                                    None, None), "mpm_frame_records")

    def partial_records(frame):
        check(LIB.mpm_frame_records(h._h, frame, 0, None, None, pv.ctypes.data, ctypes.byref(cnt[1]),
                                    jp.ctypes.data, ctypes.byref(cnt[2]), st.ctypes.data, ctypes.byref(cnt[3])),
              "mpm_frame_records")

    full_records(0)                                  # first call: the library's frame buffers
    clock("frame_full", lambda: full_records(1))
    n_full = cnt[0].value
    h.step(1000)
    clock("frame_partial", lambda: partial_records(2))
    n_part = [c.value for c in cnt[1:]]
    sens, force = h.sensors()
    out_dir = tempfile.mkdtemp(prefix="icempm_io_")
    try:
        p = h.params()
        f_full = clock("save_frame_full", lambda: snap.save_frame(out_dir, 1, p, sens, force, False,
                                                                 points=pts[:n_full]))
        f_part = clock("save_frame_partial", lambda: snap.save_frame(
            out_dir, 2, p, sens, force, True, upd_pos=pv[:n_part[0]], upd_jp=jp[:n_part[1]],
            upd_status=st[:n_part[2]]))
        down = clock("download", lambda: h.download())
        m = down.shape[1]
        host = pinned_empty((28, n))
        h.download(out=host)                         # first touch of the pages
        clock("download_pinned", lambda: h.download(out=host))
        buf = np.zeros((28, n))
        buf[:, :m] = down
        f_snap = clock("save_snapshot", lambda: snap.save_snapshot(out_dir, 3, p, buf, m, sens, compress=False))
        _, back, size, _ = clock("read_snapshot", lambda: snap.read_snapshot(f_snap))
        c = h.cohesion() if coh is not None else None    # blocks without per-particle cohesion
        clock("upload", lambda: h.upload(np.ascontiguousarray(back[:, :size]), cohesion=c))
        host[:, :size] = back[:, :size]
        clock("upload_pinned", lambda: h.upload(host[:, :size] if size == n else
                                                 np.ascontiguousarray(host[:, :size]), cohesion=c))
        sizes = {k: os.path.getsize(v) for k, v in (("frame_full", f_full), ("frame_partial", f_part),
                                                    ("snapshot", f_snap))}
    finally:
        shutil.rmtree(out_dir, ignore_errors=True)
    # the CPU restatement of the record logic on the same points
    from oracle.frames import FrameState
    fs = FrameState()
    t0 = time.perf_counter()
    fs.full(down, 1)
    cpu_full = time.perf_counter() - t0
    t0 = time.perf_counter()
    fs.partial(down, 2, p.InitialTimeStep, p.UpdateEveryNthStep, p.animation_threshold_pos)
    cpu_part = time.perf_counter() - t0
    rec_bytes = {"frame_full": n_full * snap.VISUAL_POINT.itemsize,
                 "frame_partial": n_part[0] * snap.UPDATE_POS.itemsize + n_part[1] * snap.UPDATE_JP.itemsize
                 + n_part[2] * snap.UPDATE_STATUS.itemsize, "soa": 28 * 8 * m}
    out = {"metric": "seconds", "value": t["frame_full"], "unit": "s", "n_gpus": 1, "higher_is_better": False,
           "data": "synthetic", "dtype": args.precision,
           "config": {"workload": args.workload, "particles": n, "precision": args.precision},
           "seconds": t, "records": {"full": n_full, "partial_pos": n_part[0], "partial_jp": n_part[1],
                                     "partial_status": n_part[2]},
           "bytes": rec_bytes, "file_bytes": sizes,
           "cpu_baseline": {"frame_full": cpu_full, "frame_partial": cpu_part, "unit": "s", "cores": 1,
                            "kind": "port", "sample": f"the {m} downloaded points (numpy)"}}
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.io:
        return run_io(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.adjoint:
        return run_adjoint(args)
    if args.partitions:
        return run_partitions(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
