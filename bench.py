#!/usr/bin/env python3
"""Benchmark: MTTKRP along every mode of the large skewed tensor (FP32).

Workload (one GPU): 3-mode tensor 4,800,000 x 1,800,000 x 1,800,000 built
from 140,000,000 draws per mode of Zipf(s=1.1), duplicates merged by
summing (about 100.9M nonzeros), values log-normal(0, 1) in FP32, 65 ALTO
bits (128-bit index), rank 32.  Seeded synthetic data stands in for the
FROSTT tensors the reference measures on.

A step is one MTTKRP sweep: for every mode n the output matrix is zeroed and
M_n = X_(n) (U_{others} Khatri-Rao) is computed by the ALTO kernel, the
reference's mttkrp_alto_par sweep (src/main.cpp:476-495) with fixed inputs.

  value  = nonzeros x modes / step time (device-resident inputs)   [Gnnz/s/mode]
  e2e    = the same through the drop-in host call (altob_mttkrp_sweep_host:
           host factors copied in, every mode, all factors copied back)
  roofline = algorithmic bytes of one MTTKRP launch / its CUDA-event time
  cpu_baseline = the reference's OpenMP mttkrp_alto_par on a bounded sample

--impl reference times the reference's own CPU implementation instead.

--workload batch runs the batched CP-ALS workload instead: 512 independent
tensors (order 3, 4 or 5; dims log-uniform in [100, 50,000]; nnz log-uniform
in [10,000, 2,000,000]; uniform coordinates; values uniform (0, 1]; rank from
{8, 16, 32, 64}), 25 iterations each, solved by altob_batch_cpd_als in FP32
(one step = the whole batch), beside the plain one-tensor-at-a-time FP64
altob_cpd_als path on the same tensors and initial models.

--workload serve replays a served request stream: Poisson arrivals at 200/s,
70% CP-ALS and 30% CP-APR, every tensor 4-mode 20,000 x 10,000 x 5,000 x 200
with INT32 Poisson counts from a rank-8 Gamma(0.3, 1) Kruskal model (count
total log-uniform in [50,000, 20,000,000]; CP-ALS decomposes the counts as
FP32 values), rank from {16, 32, 64}, tolerance 1e-4, at most 50 iterations,
150 GB HBM budget; FP32 served path (concurrent workers, CP-ALS batching)
beside the plain one-at-a-time FP64 path on the same stream.

--workload cpals runs CP-ALS on the same large tensor (rank 32, 10
iterations) with the FP32 model (FP64 Gram/solve/fit) and with the FP64 model
on FP64 values from the same initial factors, and reports the time per
iteration and the fit agreement.

--workload apr runs CP-APR on the 4-mode count tensor 20,000 x 10,000 x 5,000
x 200 (INT32 Poisson counts from a rank-10 Gamma(0.3, 1) Kruskal model, about
50M distinct nonzeros), rank 16, FP32 model with FP64 KKT and
log-likelihood, 50 outer x 10 inner iterations with fixed inner counts; the
metric counts one Phi pass over all nonzeros per inner iteration.  The FP64
model runs the same schedule for the agreement check, and the reference's
own cp_apr_alto (OpenMP) runs a bounded sample on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DIMS = (4_800_000, 1_800_000, 1_800_000)
DRAWS = 140_000_000
RANK = 32
ZIPF_S = 1.1
SEED = 2
METRIC = "mttkrp_gnnz_per_s_per_mode"
UNIT = "Gnnz/s/mode"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="altob", choices=["altob", "reference"])
    p.add_argument("--draws", type=int, default=DRAWS, help="Zipf draws per mode (smaller = profiling case)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-baseline", action="store_true", help=argparse.SUPPRESS)
    p.add_argument("--no-serve", action="store_true", help="default workload: skip the served-stream object")
    p.add_argument("--no-batch", action="store_true", help="default workload: skip the batched-solve object")
    p.add_argument("--no-fp64", action="store_true", help="default workload: skip the FP64 MTTKRP companion")
    p.add_argument("--cpu-iters", type=int, default=3, help=argparse.SUPPRESS)
    p.add_argument("--workload", default="mttkrp", choices=["mttkrp", "batch", "serve", "apr", "cpals"])
    p.add_argument("--apr-nnz", type=int, default=50_000_000, help="apr: target distinct nonzeros")
    p.add_argument("--apr-outer", type=int, default=50)
    p.add_argument("--serve-requests", type=int, default=60)
    p.add_argument("--serve-workers", type=int, default=4)
    p.add_argument("--serve-batch", type=int, default=32)
    p.add_argument("--serve-policy", default="fifo", choices=["fifo", "least_work"])
    p.add_argument("--batch-count", type=int, default=512)
    p.add_argument("--batch-iters", type=int, default=25)
    p.add_argument("--no-baseline", action="store_true", help="batch: skip the one-at-a-time FP64 arm")
    return p.parse_args()


# ------------------------------------------------------------ data (torch)

def zipf_tensor_torch(dims, draws, s, seed, device):
    """Config-2 tensor generated on the device (alto_b200.synth.zipf_tensor_torch)."""
    from alto_b200 import synth
    return synth.zipf_tensor_torch(dims, draws, s, seed, device)


# ------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples while the timed region runs."""

    def __init__(self):
        self.samples = []
        self.proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", "0", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], None, set()
        for p in self.samples:
            try:
                sm.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[3 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# --------------------------------------------------------- CPU baselines

def host_tensor(draws, seed):
    """The workload's tensor in host memory: (dims, cidx (3 x nnz uint64), vals
    float64, nnz, generator).  Generated on cuda:0 when a GPU is present (the
    same generator and seed as the GPU arm, so both arms see the same
    nonzeros), else by the CPU generator (same distribution, other draws)."""
    try:
        import torch
        if torch.cuda.is_available():
            cidx, vals, nnz = zipf_tensor_torch(DIMS, draws, ZIPF_S, seed, "cuda")
            hc = cidx.cpu().numpy().astype(np.uint64)
            hv = vals.double().cpu().numpy()
            del cidx, vals
            torch.cuda.empty_cache()
            return np.array(DIMS, np.uint64), hc, hv, nnz, "torch (cuda:0), as the GPU arm"
    except ImportError:
        pass
    from alto_b200 import synth
    dims, cidx, vals = synth.zipf_tensor(DIMS, draws, seed, s=ZIPF_S)
    return dims, cidx, vals.astype(np.float64), int(vals.shape[0]), "numpy (CPU generator: other draws)"


def ref_mttkrp_sweeps(draws, seed, iters):
    """The reference's mttkrp_alto_par benchmark sweep (BenchmarkAlto,
    src/main.cpp:476-495) on the workload's tensor: oracle/_ref (the
    reference compiled from its sources) with every host thread, or the
    oracle port when that library is absent.  Returns a dict."""
    from oracle import orc
    dims, cidx, vals, nnz, gen = host_tensor(draws, seed)
    if orc.ref_available():
        ref = orc.RefLib()
        cores = ref.max_threads()
        # create_alto once (untimed by the reference itself), a warm-up
        # sweep, then `iters` timed sweeps
        t, create_s = ref.bench_mttkrp(dims, cidx, vals, cores, 128, RANK, iters, seed)
        kind, march = "reference", ref.march
    else:
        o = orc.Oracle()
        at = o.create(dims, cidx, vals, 1, 128)
        U = [np.random.default_rng(m).random((int(x), RANK)) for m, x in enumerate(dims)]
        t0 = time.perf_counter()
        for _ in range(iters):
            for m in range(3):
                at.mttkrp(m, U, RANK)
        t = time.perf_counter() - t0
        create_s, kind, cores, march = 0.0, "port", 1, "gcc -O2 (oracle)"
    return {"value": nnz * 3 * iters / t / 1e9, "unit": UNIT, "cores": cores, "kind": kind, "seconds": t,
            "create_s": create_s, "nnz": nnz, "isa": orc.host_isa(), "build": march, "generator": gen,
            "sample": f"the full workload ({nnz} nonzeros from {draws} Zipf(1.1) draws per mode), rank {RANK}, "
                      f"{iters} sweeps of mttkrp_alto_par over 3 modes, FP64, 128-bit ALTO index, "
                      f"nprtn = {cores} (OpenMP threads)"}


def cpu_baseline(args):
    """The reference's sweep on the same tensor, in a child process (its
    OpenMP settings apply there only)."""
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    env["OMP_PROC_BIND"] = "close"
    env["OMP_PLACES"] = "cores"
    env["OPENBLAS_NUM_THREADS"] = "1"
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-baseline", "--draws", str(args.draws),
                        "--cpu-iters", str(args.cpu_iters)], env=env, capture_output=True, text=True, timeout=1500)
    line = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode != 0 or not line:
        return {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                "sample": "failed: " + (r.stderr[-300:] if r.stderr else "no output")}
    return json.loads(line[-1])


def sub_workload(args, workload, extra=()):
    """Runs `bench.py --workload <w>` in a child process (the GPU to itself)
    and returns its JSON line, or an error record."""
    cmd = [sys.executable, os.path.abspath(__file__), "--workload", workload, "--steps", str(min(args.steps, 3)),
           "--warmup", str(min(args.warmup, 3))] + list(extra)
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=1200)
    except subprocess.TimeoutExpired:
        return {"error": "timeout"}
    line = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode != 0 or not line:
        return {"error": (r.stderr[-400:] if r.stderr else "no output")}
    return json.loads(line[-1])


# ------------------------------------------------------------ arms

def rank_seed(base, rank):
    """Seed of rank `rank`'s replica (weak scaling: every rank its own data)."""
    return base + 7919 * rank


def max_over_ranks(value, dist=None, device="cpu"):
    """The job time of a replicated run: the slowest rank's (all-reduce MAX)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    r = ref_mttkrp_sweeps(args.draws, SEED, args.steps)
    value = r["value"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["seconds"] / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, r["nnz"], 65, 128, ws),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "isa": r["isa"], "build": r["build"], "sample": r["sample"]},
            "create_s": r["create_s"], "generator": r["generator"],
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args, nnz, alto_bits, lit_bits, ws):
    return {"workload": "mttkrp_sweep_zipf3_4.8Mx1.8Mx1.8M" if args.draws == DRAWS else
            f"mttkrp_sweep_zipf3_small_{args.draws}", "dims": list(DIMS), "draws": args.draws, "nnz": nnz,
            "rank": RANK, "alto_bits": alto_bits, "lit_bits": lit_bits, "parallelism": f"replicas{ws}",
            "l2": "inputs larger than L2 (no flush)"}


def run_altob(args):
    import torch
    import alto_b200 as ab

    ws, rank, local = dist_setup()
    # the batched and served objects first, each in a child process with the
    # GPU to itself (no context of this process on the device yet)
    batch = serve = None
    if rank == 0 and ws == 1 and args.draws == DRAWS:
        if not args.no_batch:
            batch = sub_workload(args, "batch")
        if not args.no_serve:
            serve = sub_workload(args, "serve")
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    # per-rank data: replicas of the workload with rank-dependent seeds (weak scaling)
    cidx, vals, nnz = zipf_tensor_torch(DIMS, args.draws, ZIPF_S, rank_seed(SEED, rank), dev)
    at = ab.create_alto_device(3, np.array(DIMS, np.uint64), nnz, cidx, vals, nprtn=1024, lit_bits=128,
                               val_dtype="f32", stream=stream)
    if args.no_fp64:
        del cidx, vals
    torch.cuda.synchronize()
    torch.cuda.empty_cache()  # the generator's temporaries: a profiler saves every allocation
    info = at.info()
    g = torch.Generator(device=dev)
    g.manual_seed(SEED)
    U = [torch.rand(d, RANK, dtype=torch.float32, device=dev, generator=g) for d in DIMS]
    out = [torch.zeros(d, RANK, dtype=torch.float32, device=dev) for d in DIMS]

    def ptrs_for(n):
        return [out[m] if m == n else U[m] for m in range(3)]

    evs = [[torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)] for _ in range(3 * args.steps)]

    def step(k=None):
        for n in range(3):
            out[n].zero_()
            if k is not None:
                evs[3 * k + n][0].record(stream)
            ab.mttkrp_alto_par(n, ptrs_for(n), RANK, at, algo="auto", accumulate=True, stream=stream)
            if k is not None:
                evs[3 * k + n][1].record(stream)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    clk = ClockSampler()
    clk.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        step(k)
    t1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = t0.elapsed_time(t1)
    clocks = clk.stop()
    at_plan_modes = at.info()["plan_modes"]
    free_b, total_b = torch.cuda.mem_get_info(dev)
    dev_used_gb = (total_b - free_b) / 1e9  # the whole process's device memory after the timed steps
    ms = max_over_ranks(ms, dist, dev)
    ms_step = ms / args.steps
    value = ws * nnz * 3 / (ms_step / 1e3) / 1e9

    # roofline of the MTTKRP kernel: algorithmic bytes per launch
    stream_b = nnz * (info["key_bytes"] + 4)  # index words as stored on the device + FP32 value
    fac_b = [d * RANK * 4 for d in DIMS]
    launch_ms = [[], [], []]
    for k in range(args.steps):
        for n in range(3):
            launch_ms[n].append(evs[3 * k + n][0].elapsed_time(evs[3 * k + n][1]))
    bytes_per_mode = [stream_b + sum(fac_b) for n in range(3)]  # other factors read once + output written once
    avg_ms = [statistics.mean(x) for x in launch_ms]
    achieved = sum(bytes_per_mode) / (sum(avg_ms) / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = l2 = l1p = None
    tf = os.path.join(ROOT, "profiles", "mttkrp_traffic.json")
    if os.path.exists(tf):
        try:
            with open(tf) as f:
                tj = json.load(f)
            traffic = tj.get("per_launch_bytes_full_size")
            l2 = tj.get("l2")
            l1p = tj.get("l1_pipe")
        except (OSError, ValueError):
            traffic = l2 = l1p = None
    # the gather ceiling: the L1 data pipe retires one wavefront per SM cycle
    # and the kernel needs wavefronts_per_nnz of them per nonzero (measured)
    ceiling = None
    if l1p and args.draws == DRAWS:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
        floor_ms = nnz * l1p["wavefronts_per_nnz"] / (sms * mhz * 1e6) * 1e3
        ceiling = {"bound": "l1 data pipe (factor-row gathers)", "wavefronts_per_nnz": l1p["wavefronts_per_nnz"],
                   "sms": sms, "sm_mhz": mhz, "floor_ms_per_launch": floor_ms,
                   "frac": floor_ms / statistics.mean(avg_ms), "source": l1p["from"]}

    e2e = None
    if not args.no_e2e:
        hU = [torch.empty(d, RANK, dtype=torch.float32, pin_memory=True) for d in DIMS]
        for h, u in zip(hU, U):
            h.copy_(u.cpu())
        hU_np = [h.numpy() for h in hU]
        init_np = [h.copy() for h in hU_np]

        def e2e_step():
            # the reference's benchmark loop (src/main.cpp:476-495) through the
            # drop-in: host factors copied in once, += MTTKRP on every mode,
            # all factors copied back
            ab.mttkrp_sweep_host(at, hU_np, RANK, iters=1, stream=stream)

        e2e_step()  # warm-up (also sizes the handle's scratch)
        torch.cuda.synchronize()
        ke = max(2, min(args.steps, 5))
        te = 0.0
        for _ in range(ke):
            for h, h0 in zip(hU_np, init_np):  # untimed: keep the factors bounded
                np.copyto(h, h0)
            tA = time.perf_counter()
            e2e_step()
            torch.cuda.synchronize()
            te += time.perf_counter() - tA
        te /= ke
        h2d = sum(fac_b)
        d2h = sum(fac_b)
        e2e = {"value": ws * nnz * 3 / te / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": te * 1e3, "steps": ke,
               "api": "altob_mttkrp_sweep_host (the reference's mttkrp_alto_par benchmark sweep with host "
                      "factors: copied in once, every mode, copied out)"}

    # same-precision companion: FP64 values and factors, the reference's
    # arithmetic, on the same nonzeros (device-resident, CUDA events)
    f64 = None
    if not args.no_fp64:
        del out
        at64 = ab.create_alto_device(3, np.array(DIMS, np.uint64), nnz, cidx, vals.double(), nprtn=1024,
                                     lit_bits=128, val_dtype="f64", stream=stream)
        del cidx, vals
        U64 = [u.double() for u in U]
        o64 = [torch.zeros(d, RANK, dtype=torch.float64, device=dev) for d in DIMS]

        def step64():
            for n in range(3):
                o64[n].zero_()
                ab.mttkrp_alto_par(n, [o64[m] if m == n else U64[m] for m in range(3)], RANK, at64, algo="auto",
                                   accumulate=True, stream=stream)

        for _ in range(3):
            step64()
        k64 = max(3, min(args.steps, 10))
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        f0.record(stream)
        for _ in range(k64):
            step64()
        f1.record(stream)
        torch.cuda.synchronize()
        ms64 = f0.elapsed_time(f1) / k64
        b64 = nnz * (info["key_bytes"] + 8) + sum(d * RANK * 8 for d in DIMS)
        f64 = {"value": ws * nnz * 3 / (ms64 / 1e3) / 1e9, "unit": UNIT, "ms_per_step": ms64, "steps": k64,
               "dtype": "f64", "algorithmic_bytes_per_launch": b64,
               "roofline_frac": 3 * b64 / (ms64 / 1e3) / 1e9 / peak,
               "what": "the same sweep with FP64 values and factors (the reference's arithmetic), same nonzeros"}
        del at64, U64, o64
    else:
        del out
    del at, U
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and not args.no_cpu and ws == 1:
        cpu = cpu_baseline(args)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": workload_config(args, nnz, info["alto_bits"], info["lit_bits"], ws),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                             "kernel": "k_planned (MTTKRP, tile plans)" if at_plan_modes == 7 else "k_grouped (MTTKRP)", "launch_ms_per_mode": avg_ms,
                             "algorithmic_bytes_per_launch": bytes_per_mode,
                             "traffic_source": "profiles/mttkrp_traffic.json (two small captures, extrapolated)",
                             "l2": l2, "ceiling": ceiling},
                "e2e": e2e, "gpu_launches": 3 * args.steps, "clocks": clocks, "cpu_baseline": cpu,
                "device_mem_used_gb": dev_used_gb,
                "fp64": f64, "batch": batch, "serve": serve}
        print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """Batched CP-ALS workload (see the module docstring)."""
    import torch
    import alto_b200 as ab
    from alto_b200 import synth

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    iters = args.batch_iters
    shapes = synth.batch_shapes(args.batch_count, SEED + 31 * rank)
    t32, t64, init = [], [], []
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + rank)
    for k, (dims, nnz, r) in enumerate(shapes):
        cidx, vals = synth.uniform_coo_torch(dims, nnz, SEED * 1000 + k + 7919 * rank, dev)
        d = np.array(dims, np.uint64)
        t32.append(ab.create_alto_device(len(dims), d, nnz, cidx, vals.float(), nprtn=128, lit_bits=0,
                                         val_dtype="f32", stream=stream))
        if not args.no_baseline:
            t64.append(ab.create_alto_device(len(dims), d, nnz, cidx, vals, nprtn=128, lit_bits=0,
                                             val_dtype="f64", stream=stream))
        init.append([torch.rand(int(x), r, dtype=torch.float64, device=dev, generator=g) for x in dims])
        del cidx, vals
    torch.cuda.synchronize()
    nnz_total = sum(s[1] for s in shapes)
    M32 = [ab.KruskalModel(list(s[0]), s[2], [u.float() for u in init[k]],
                           torch.ones(s[2], dtype=torch.float32, device=dev)) for k, s in enumerate(shapes)]

    def reset32():
        for k, m in enumerate(M32):
            for u, u0 in zip(m.U, init[k]):
                u.copy_(u0)

    b = ab.BatchCPD(t32, M32, fit_capacity=iters, stream=stream)
    ta = time.perf_counter()
    b.autotune(stream=stream)
    tune_s = time.perf_counter() - ta
    for _ in range(max(1, min(args.warmup, 3))):
        reset32()
        b.solve(iters, 0.0, stream=stream)
    reset32()
    torch.cuda.synchronize()
    clk = ClockSampler()
    clk.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(1, min(args.steps, 3))
    ms_all = []
    for _ in range(steps):
        reset32()
        e0.record(stream)
        fits32, its32 = b.solve(iters, 0.0, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_all.append(e0.elapsed_time(e1))
    clocks = clk.stop()
    desc = b.describe()
    launches_iter = int(desc.split("launches_per_iteration=")[1].split()[0])
    ms = statistics.median(ms_all)
    value = args.batch_count / (ms / 1e3)

    # cost of a replayed iteration in which every tensor has stopped (each
    # kernel of the graph launches and finds no active tensor): solves of 2
    # and 5 iterations with a tolerance every tensor meets after its second
    # fit differ by three such replays (each length run twice: the second
    # run replays the graph captured by the first)
    idle = {}
    for n_it in (2, 2, 5, 5):
        reset32()
        e0.record(stream)
        b.solve(n_it, 1e300, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        idle[n_it] = e0.elapsed_time(e1)
    idle_ms = (idle[5] - idle[2]) / 3

    base = None
    fit_err = None
    if not args.no_baseline:
        M64 = [ab.KruskalModel(list(s[0]), s[2], [u.clone() for u in init[k]],
                               torch.ones(s[2], dtype=torch.float64, device=dev)) for k, s in enumerate(shapes)]
        ab.cpd_alto(t64[0], ab.KruskalModel(list(shapes[0][0]), shapes[0][2], [u.clone() for u in init[0]],
                                            torch.ones(shapes[0][2], dtype=torch.float64, device=dev)), 2, 0.0)
        torch.cuda.synchronize()
        f64 = []
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for k in range(len(shapes)):
            f64.append(ab.cpd_alto(t64[k], M64[k], iters, 0.0))
        b1.record(stream)
        torch.cuda.synchronize()
        bms = b0.elapsed_time(b1)
        base = {"value": args.batch_count / (bms / 1e3), "unit": "solves/s", "ms": bms,
                "path": "altob_cpd_als, FP64 model and values, one tensor after another on one stream"}
        fd = [abs(fits32[k][iters - 1] - f64[k][-1]) for k in range(len(shapes))]
        fit_err = {"final_within_tol": int(sum(d < 1e-4 for d in fd)), "of": len(fd),
                   "final_median_abs": float(np.median(fd)),
                   "final_max_abs": float(max(fd)),
                   "all_iters_max_abs": float(max(np.max(np.abs(fits32[k][:iters] - f64[k])) for k in
                                                  range(len(shapes)))),
                   "tolerance": 1e-4}
    b.close()
    line = {"metric": "batched_cpals_solves_per_s", "value": value, "unit": "solves/s", "n_gpus": ws,
            "steps": steps, "warmup": max(1, min(args.warmup, 3)), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 Gram/solve/fit)", "data": "synthetic",
            "config": {"workload": f"batched_cpals_{args.batch_count}x{iters}it", "tensors": args.batch_count,
                       "iterations": iters, "nnz_total": nnz_total,
                       "orders": dict((o, sum(1 for s in shapes if len(s[0]) == o)) for o in (3, 4, 5)),
                       "ranks": dict((r, sum(1 for s in shapes if s[2] == r)) for r in (8, 16, 32, 64))},
            "baseline_fp64_one_at_a_time": base,
            "speedup_vs_fp64_one_at_a_time": (value / base["value"]) if base else None,
            "fit_vs_fp64": fit_err, "autotune_s": tune_s, "schedule": desc,
            "launches_per_iteration": launches_iter,
            "idle_iteration_ms": idle_ms,
            "idle_iteration_what": "a replayed iteration whose kernels all find their tensors stopped: "
                                   "launch and scheduling cost of the graph, against ms_per_step / iterations",
            "gpu_launches": steps * (1 + iters * launches_iter), "clocks": clocks,
            "nnz_mode_rate_gnnz_s": sum(s[1] * len(s[0]) for s in shapes) * iters / (ms / 1e3) / 1e9}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """Served decomposition stream (see the module docstring)."""
    import torch
    import alto_b200 as ab
    from alto_b200 import serve, synth

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = synth.served_stream(args.serve_requests, SEED + 17 * rank)
    inputs = []
    for k, (at, kind, dims, nnz, r, seed) in enumerate(stream):
        cidx, cnt = synth.poisson_kruskal_torch(dims, 8, nnz, seed, dev)
        if kind == "als":
            inputs.append((kind, dims, cidx, cnt.float(), cnt.double(), r, seed))
        else:
            inputs.append((kind, dims, cidx, cnt, cnt, r, seed))
    torch.cuda.synchronize()
    arrivals = [x[0] for x in stream]

    def requests(ftype):
        out = []
        for kind, dims, cidx, v32, v64, r, seed in inputs:
            vals = v32 if ftype == ab.F32 else v64
            k = serve.ALS if kind == "als" else serve.APR
            req = serve.Server.make_request(k, dims, cidx, vals, r, 50, 1e-4, seed, ftype, max_inner=10)
            out.append((req, (cidx, vals)))
        return out

    # served path; a short warm-up stream first tunes the shape classes
    srv = serve.Server(hbm_budget_gb=150, workers=args.serve_workers, max_batch=args.serve_batch,
                       policy=args.serve_policy)
    reqs = requests(ab.F32)
    nw = min(len(reqs), 12)
    serve.replay(srv, reqs[:nw], [0.0] * nw)
    clk = ClockSampler()
    clk.start()
    time.sleep(0.3)
    res, summ = serve.replay(srv, reqs, arrivals)
    clocks = clk.stop()
    for kind in ("als", "apr"):
        lat = [r["latency"] for (k, *_), r in zip(inputs, res) if k == kind]
        summ[f"{kind}_p50_ms"] = float(np.percentile(lat, 50) * 1e3) if lat else None
        summ[f"{kind}_iters_mean"] = float(np.mean([r["iters"] for (k, *_), r in zip(inputs, res) if k == kind])) \
            if lat else None
    peak = srv.stats()["peak_bytes"]
    srv.close()
    base = None
    agree = None
    if not args.no_baseline:
        srv = serve.Server(hbm_budget_gb=150, workers=1, max_batch=1, plain=True, policy="fifo")
        bres, bsumm = serve.replay(srv, requests(ab.F64), arrivals)
        srv.close()
        base = dict(bsumm, path="plain one-at-a-time FP64: altob_cpd_als / altob_cp_apr, one worker, no batching")
        for kind in ("als", "apr"):
            base[f"{kind}_service_s"] = float(sum(b["t_end"] - b["t_start"] for (k, *_), b in zip(inputs, bres)
                                                  if k == kind))
        als_d = [abs(a["fit"] - b["fit"]) for (kind, *_), a, b in zip(inputs, res, bres) if kind == "als"]
        apr_d = [abs(a["loglik"] - b["loglik"]) / max(1e-300, abs(b["loglik"]))
                 for (kind, *_), a, b in zip(inputs, res, bres) if kind == "apr"]
        agree = {"als_fit_within_1e-4": int(sum(d < 1e-4 for d in als_d)), "als": len(als_d),
                 "als_fit_max_abs": float(max(als_d)) if als_d else None,
                 "als_fit_median_abs": float(np.median(als_d)) if als_d else None,
                 "apr_loglik_within_1e-4_rel": int(sum(d < 1e-4 for d in apr_d)), "apr": len(apr_d),
                 "apr_loglik_max_rel": float(max(apr_d)) if apr_d else None}
    line = {"metric": "served_solves_per_s", "value": summ["solves_per_s"], "unit": "solves/s", "n_gpus": ws,
            "steps": 1, "warmup": 1, "ms_per_step": summ["makespan_s"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 Gram/solve/fit/KKT/LL)",
            "data": "synthetic",
            "config": {"workload": f"served_stream_{len(inputs)}req_200rps", "requests": len(inputs),
                       "als": sum(1 for x in inputs if x[0] == "als"), "apr": sum(1 for x in inputs if x[0] == "apr"),
                       "nnz_total": int(sum(int(x[3].shape[0]) for x in inputs)), "hbm_budget_gb": 150,
                       "workers": args.serve_workers, "max_batch": args.serve_batch,
                       "policy": args.serve_policy},
            "served": summ, "peak_admitted_bytes": peak, "baseline_fp64_one_at_a_time": base,
            "speedup_vs_fp64_one_at_a_time": (summ["solves_per_s"] / base["solves_per_s"]) if base else None,
            "agreement_vs_fp64": agree, "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_cpals(args):
    """CP-ALS on the large skewed tensor (see the module docstring)."""
    import torch
    import alto_b200 as ab

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    iters = 10
    cidx, vals, nnz = zipf_tensor_torch(DIMS, args.draws, ZIPF_S, rank_seed(SEED, rank), dev)
    d = np.array(DIMS, np.uint64)
    at32 = ab.create_alto_device(3, d, nnz, cidx, vals, nprtn=1024, lit_bits=128, val_dtype="f32")
    at64 = None if args.no_baseline else ab.create_alto_device(3, d, nnz, cidx, vals.double(), nprtn=1024,
                                                                lit_bits=128, val_dtype="f64")
    del cidx, vals
    g = torch.Generator(device=dev)
    g.manual_seed(SEED)
    init = [torch.rand(x, RANK, dtype=torch.float64, device=dev, generator=g) for x in DIMS]

    def model(dt):
        return ab.KruskalModel(list(DIMS), RANK, [u.to(dt).clone() for u in init],
                               torch.ones(RANK, dtype=dt, device=dev))

    ab.cpd_alto(at32, model(torch.float32), 1, 0.0)  # warm-up
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    clk = ClockSampler()
    clk.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    f32 = ab.cpd_alto(at32, model(torch.float32), iters, 0.0)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms32 = e0.elapsed_time(e1)
    f64, ms64 = None, None
    if at64 is not None:
        e0.record(stream)
        f64 = ab.cpd_alto(at64, model(torch.float64), iters, 0.0)
        e1.record(stream)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1)
    line = {"metric": "cpals_ms_per_iteration", "value": ms32 / iters, "unit": "ms", "n_gpus": ws, "steps": iters,
            "warmup": 1, "ms_per_step": ms32 / iters, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 Gram/solve/fit)", "data": "synthetic",
            "config": {"workload": "cpals_zipf3_4.8Mx1.8Mx1.8M", "dims": list(DIMS), "nnz": nnz, "rank": RANK,
                       "iterations": iters, "alto_bits": 65},
            "mttkrp_gnnz_per_s_per_mode_in_solve": nnz * 3 * iters / (ms32 / 1e3) / 1e9,
            "fits_fp32": list(map(float, f32)), "fits_fp64": list(map(float, f64)) if f64 is not None else None,
            "fp64_ms_per_iteration": ms64 / iters if ms64 else None,
            "fit_max_abs_diff_fp32_vs_fp64": float(np.max(np.abs(np.array(f32) - np.array(f64))))
            if f64 is not None else None, "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_apr(args):
    """CP-APR workload (see the module docstring)."""
    import torch
    import alto_b200 as ab
    from alto_b200 import synth

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dims = synth.CONFIG3_DIMS
    R, inner, outer = 16, 10, args.apr_outer
    total = args.apr_nnz
    cidx, cnt = synth.poisson_kruskal_torch(dims, 10, total, SEED + 3 + 101 * rank, dev, shape=0.3)
    if cnt.shape[0] < 0.97 * args.apr_nnz:  # more draws to reach the distinct-nonzero target
        total = int(total * args.apr_nnz / cnt.shape[0] * 1.02)
        del cidx, cnt
        cidx, cnt = synth.poisson_kruskal_torch(dims, 10, total, SEED + 3 + 101 * rank, dev, shape=0.3)
    nnz = int(cnt.shape[0])
    at = ab.create_alto_device(4, np.array(dims, np.uint64), nnz, cidx, cnt, nprtn=1024, lit_bits=0, val_dtype="u32")
    del cidx
    g = torch.Generator(device=dev)
    g.manual_seed(SEED)
    init = [torch.rand(d, R, dtype=torch.float64, device=dev, generator=g) for d in dims]

    def model(dt):
        return ab.KruskalModel(list(dims), R, [u.to(dt).clone() for u in init], torch.ones(R, dtype=dt, device=dev))

    # warm-up: a short solve loads every kernel of the path
    ab.cp_apr_alto(at, model(torch.float32), 2, 2, epsilon=0.0, dobench=True)
    torch.cuda.synchronize()
    clk = ClockSampler()
    clk.start()
    time.sleep(0.3)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    r32 = ab.cp_apr_alto(at, model(torch.float32), outer, inner, epsilon=0.0, dobench=True)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    passes = r32["inner"]  # Phi passes over all nonzeros
    value = nnz * passes / (ms / 1e3) / 1e9
    r64 = None
    if not args.no_baseline:
        e0.record(stream)
        r64 = ab.cp_apr_alto(at, model(torch.float64), outer, inner, epsilon=0.0, dobench=True)
        e1.record(stream)
        torch.cuda.synchronize()
        r64 = dict(r64, ms=e0.elapsed_time(e1))
    cpu = None
    if not args.no_cpu and rank == 0:
        from oracle import orc
        sample = 2_000_000
        sc, sv = synth.poisson_kruskal_torch(dims, 10, sample, SEED + 33, dev, shape=0.3)
        sc, sv = sc.cpu().numpy().astype(np.uint64), sv.cpu().numpy().astype(np.float64)
        so, si = 2, 10
        t0 = time.perf_counter()
        if orc.ref_available():
            ref = orc.RefLib()
            _, _, rs = ref.apr(np.array(dims, np.uint64), sc, sv, ref.max_threads(), 64, R, so, si, 0.0, 1e-10,
                               1e-10, 1e-2, True, 1)
            kind, cores = "reference", ref.max_threads()
        else:
            o = orc.Oracle()
            ot = o.create(np.array(dims, np.uint64), sc, sv, 1, 64)
            U, lam = o.random_init(np.array(dims, np.uint64), R, 1)
            rs = ot.cp_apr(U, lam, R, so, si, eps=0.0, dobench=True)
            kind, cores = "port", 1
        t = time.perf_counter() - t0
        cpu = {"value": len(sv) * rs["inner"] / t / 1e9, "unit": "Gnnz/s", "cores": cores, "kind": kind,
               "seconds": t, "sample": f"{len(sv)} nonzeros of the same distribution (2M Poisson draws), rank {R}, "
                                       f"{so} outer x {si} inner iterations of cp_apr_alto, FP64, create included"}
    line = {"metric": "cp_apr_phi_gnnz_per_s", "value": value, "unit": "Gnnz/s", "n_gpus": ws, "steps": 1,
            "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (FP64 KKT/LL)", "data": "synthetic",
            "config": {"workload": "cp_apr_4mode_20000x10000x5000x200", "dims": list(dims), "nnz": nnz,
                       "poisson_draws": total, "rank": R, "outer": outer, "inner": inner, "fixed_inner": True},
            "result_fp32": r32, "result_fp64": r64,
            "loglik_rel_diff_fp32_vs_fp64": (abs(r32["loglik"] - r64["loglik"]) / abs(r64["loglik"])) if r64 else None,
            "ms_per_outer_iteration": ms / max(1, r32["outer"]), "clocks": clocks, "cpu_baseline": cpu}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.cpu_baseline:
        print(json.dumps(ref_mttkrp_sweeps(args.draws, SEED, args.cpu_iters)), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "apr":
        return run_apr(args)
    if args.workload == "cpals":
        return run_cpals(args)
    return run_altob(args)


if __name__ == "__main__":
    sys.exit(main())
