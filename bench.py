"""Benchmark: fold-3 reproBLAS_ddot at N = 2^28 (FP64), the reproducible binned dot product.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one reproducible dot product of two 2^28-element FP64 vectors (uniform(-1,1),
seeded). Prints ONE JSON line on rank 0.

  value   device throughput in GB/s of algorithmic traffic (16 B per element), inputs
          resident in HBM, timed with CUDA events over exactly K launches of
          binnedBLAS_dbddot (2 x 2 GiB inputs, far larger than the 126 MB L2, so no flush
          is needed between steps); whole job = sum over ranks / max rank time.
  e2e     the same metric through the reference-facing call reproBLAS_rddot with pinned
          HOST buffers: every step copies the 4 GiB of inputs to the GPU (staged chunks
          overlapped with the kernels) and reads the 8-byte result back.
  roofline  the dominant kernel (the ddot reduction): algorithmic bytes per launch over
          its mean CUDA-event duration, against the measured HBM copy bandwidth.
  cpu_baseline  the ReproBLAS reference library (oracle/_ref, compiled from its own
          sources) on this host's cores: contiguous chunks, one thread each calling
          binnedBLAS_dbddot, merged with binned_dbdbadd (the reference's own MPI pattern),
          bit-identical to the single call (best of 5); one_core: reproBLAS_rddot exactly
          as shipped, single-threaded (best of 5).
  headline  last on the line: the dgemm half of the metric (plain vs int8-sliced TFLOP/s,
          error over binned_dbbound), the measured deposit ceiling, dgemv and batched.

--impl reference times that reference CPU path alone (rank 0; other ranks exit).
Multi-GPU (torchrun, --gpus N): weak scaling, each rank reduces its own 2^28 shard; the
per-rank binned states (48 bytes) are all-gathered over NCCL and merged on every GPU.
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
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "ddot GB/s (% HBM peak) at N=2^28 fold 3"
FOLD = 3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--log2n", type=int, default=28)
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-secondary", action="store_true",
                   help="skip the dgemm (plain vs int8-sliced) and dgemv measurements")
    p.add_argument("--profile-kernel", choices=["int8", "plain_gemm", "gemv_n", "gemv_t", "zdotc",
                                                "zsum", "csum", "dnrm2", "batched", "sgemv_n",
                                                "sgemv_t", "zgemv_n", "zgemv_c", "cgemv_n",
                                                "cgemv_c", "sgemm", "zgemm", "cgemm"],
                   help="only run that kernel `--steps` times on an n^3 (or n^2) case, for ncu")
    p.add_argument("--profile-n", type=int, default=2048)
    p.add_argument("--profile-m", type=int, default=0,
                   help="rows of A for the gemv profile cases (default: --profile-n)")
    p.add_argument("--profile-slices", type=int, default=7)
    p.add_argument("--sweep", action="store_true",
                   help="only run the BLAS1 sweep (N = 2^10..2^28 in powers of 4, folds 2/3/4, "
                        "four value distributions) and print its JSON table")
    return p.parse_args()


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def make_inputs(n, rank):
    rng = np.random.default_rng(2024 + rank)
    x = rng.uniform(-1.0, 1.0, n)
    y = rng.uniform(-1.0, 1.0, n)
    return x, y


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [v.strip() for v in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_dot(R, x, y, threads):
    """Reference binnedBLAS_dbddot over `threads` contiguous chunks in parallel (ctypes
    releases the GIL), merged with binned_dbdbadd. Returns (seconds, state)."""
    from _ffi import ptr, binned_zeros
    n = len(x)
    bounds = np.linspace(0, n, threads + 1).astype(np.int64)
    states = [binned_zeros(FOLD) for _ in range(threads)]
    xs = x.ctypes.data
    ys = y.ctypes.data
    import ctypes

    def work(i):
        a, b = int(bounds[i]), int(bounds[i + 1])
        R.dbddot(FOLD, b - a, ctypes.c_void_p(xs + 8 * a), 1, ctypes.c_void_p(ys + 8 * a), 1,
                 ptr(states[i]))

    R.dbdsum(FOLD, 1, ptr(np.zeros(1)), 1, ptr(binned_zeros(FOLD)))   # builds the bins table
    t0 = time.perf_counter()
    ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    total = binned_zeros(FOLD)
    for s in states:
        R.dbdbadd(FOLD, ptr(s), ptr(total))
    dt = time.perf_counter() - t0
    return dt, total


def workload_config(log2n):
    """The workload's config (identical in both arms)."""
    n = 1 << log2n
    return {"workload": "reproBLAS_ddot fold 3, N=2^%d FP64 per GPU" % log2n,
            "n_per_gpu": n, "fold": FOLD, "l2": "inputs 4 GiB >> 126 MB L2, no flush",
            "parallelism": "weak: shard per GPU, NCCL all-gather of 48-byte states"}


def cpu_reference_rddot_1core(R, x, y, reps):
    """The reference's reproBLAS_rddot exactly as shipped (single-threaded): best time of
    `reps` calls after one warm-up call, and the result."""
    from _ffi import ptr
    n = len(x)
    res = R.rddot(FOLD, n, ptr(x), 1, ptr(y), 1)
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        res = R.rddot(FOLD, n, ptr(x), 1, ptr(y), 1)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    return best, res


def reference_arm(args, rank):
    from _ffi import ref
    if rank != 0:
        return
    R = ref()
    if R is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libreproblas_ref.so "
                          "not built (make -C oracle ref needs the ReproBLAS source tree)"}))
        return
    n = 1 << args.log2n
    x, y = make_inputs(n, 0)
    threads = host_threads()
    for _ in range(max(1, min(args.warmup, 2))):
        cpu_reference_dot(R, x, y, threads)
    times = [cpu_reference_dot(R, x, y, threads)[0] for _ in range(args.steps)]
    t = min(times)
    gbs = 16.0 * n / t / 1e9
    print(json.dumps({
        "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic uniform(-1,1), seed 2024",
        "config": workload_config(args.log2n),
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference",
                         "sample": "full workload; %d threads each calling binnedBLAS_dbddot on a "
                                   "contiguous chunk, merged with binned_dbdbadd; best of %d steps"
                                   % (threads, args.steps)},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def ours_arm(args, rank, world, local_rank):
    import torch
    import reproblas_b200 as rb
    from _ffi import ptr as nptr
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    n = 1 << args.log2n
    x, y = make_inputs(n, rank)
    X = torch.from_numpy(x).cuda()
    Y = torch.from_numpy(y).cuda()
    Z = torch.zeros(2 * FOLD, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rb.call("rb_set_stream", stream.cuda_stream)

    def step():
        Z.zero_()
        rb.call("binnedBLAS_dbddot", FOLD, n, X, 1, Y, 1, Z)

    def combine():
        # exchange the 48-byte per-rank states over NCCL and merge them on every GPU
        from reproblas_b200.distributed import allgather_merge
        return allgather_merge(Z, FOLD)

    for _ in range(args.warmup):
        step()
        if world > 1:
            combine()
    torch.cuda.synchronize()
    launches0 = rb.lib.rb_kernel_launch_count()
    clocks = ClockSampler(local_rank)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
        if world > 1:
            combine()
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = rb.lib.rb_kernel_launch_count() - launches0
    total_ms = t_start.elapsed_time(t_end)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = 16.0 * n * world / (ms_per_step * 1e-3) / 1e9
    kernel_mean_ms = statistics.mean(kern_ms)
    achieved = 16.0 * n / (kernel_mean_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()

    # result parity: the GPU state equals the reference CPU state (checked below on rank 0)
    gpu_state = Z.cpu().numpy().copy()

    # e2e: reference-facing call with pinned host buffers
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.from_numpy(y).pin_memory()
    e2e_val = None
    e2e_ms = None
    res = None
    if args.e2e_steps > 0:
        res = rb.call("reproBLAS_rddot", FOLD, n, xp, 1, yp, 1)   # warm the staging ring
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            res = rb.call("reproBLAS_rddot", FOLD, n, xp, 1, yp, 1)
        t1 = time.perf_counter()
        e2e_ms = (t1 - t0) * 1e3 / args.e2e_steps
        if world > 1:
            t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e_val = 16.0 * n * world / (e2e_ms * 1e-3) / 1e9

    cpu = None
    bit_identical = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from _ffi import ref, port
        R = ref()
        kind = "reference"
        if R is None:
            R = port()
            kind = "port"
        threads = host_threads()
        cpu_reference_dot(R, x[: 1 << 20], y[: 1 << 20], threads)   # warm-up
        times = []
        state = None
        for _ in range(5):
            dt, state = cpu_reference_dot(R, x, y, threads)
            times.append(dt)
        cpu_gbs = 16.0 * n / min(times) / 1e9
        bit_identical = bool(state.tobytes() == gpu_state.tobytes())
        t1, r1 = cpu_reference_rddot_1core(R, x, y, 5)
        cpu = {"value": round(cpu_gbs, 3), "unit": "GB/s", "cores": threads, "kind": kind,
               "sample": "full N=2^%d workload, %d threads (contiguous chunks + binned_dbdbadd), "
                         "best of 5" % (args.log2n, threads),
               "bit_identical_to_gpu": bit_identical,
               "one_core": {"value": round(16.0 * n / t1 / 1e9, 3), "unit": "GB/s", "cores": 1,
                            "api": "reproBLAS_rddot as shipped (single-threaded), best of 5",
                            "ms": round(t1 * 1e3, 2),
                            "result_equals_gpu": bool(res is None or r1 == res)}}

    sec = None
    if rank == 0 and world == 1 and not args.no_secondary:
        sec = secondary(args)

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic uniform(-1,1), seed 2024+rank (host-generated)",
        "config": workload_config(args.log2n),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                     "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                     "kernel": "rb::blas1_kernel<double,3,kOpDot,vec>",
                     "kernel_ms": round(kernel_mean_ms, 5)},
        "clocks": clk,
        "gpu_launches": int(launches),
        "e2e": {"value": round(e2e_val, 3) if e2e_val else None, "unit": "GB/s",
                "h2d_bytes_per_step": 16 * n, "d2h_bytes_per_step": 8,
                "ms_per_step": round(e2e_ms, 3) if e2e_ms else None,
                "api": "reproBLAS_rddot(3, N, pinned host X, 1, pinned host Y, 1)"},
        "cpu_baseline": cpu,
        "result": res,
        "secondary": sec,
        # last on the line: the compact second half of the headline metric (dgemm plain vs
        # int8-sliced) and the dgemv fractions
        "headline": headline(sec),
    }
    traffic = os.path.join(ROOT, "profiles", "ddot_traffic.json")
    if os.path.exists(traffic):
        try:
            with open(traffic) as f:
                line["roofline"]["traffic"] = json.load(f)["bytes_per_launch_at_2^28"]
        except Exception:
            pass
    print(json.dumps(line))


def headline(sec):
    """dgemm TFLOP/s (plain binned vs int8-sliced, with error over binned_dbbound) and the
    dgemv fractions of the HBM peak, compact."""
    if not sec:
        return None
    h = {"dgemm_plain_tflops": {k: sec[k]["tflops"] for k in ("dgemm_plain_2048", "dgemm_plain_8192")
                                if k in sec}}
    if "fp64_probe" in sec:
        h["dgemm_ceiling_tflops"] = sec["fp64_probe"]["dgemm_ceiling_tflops"]
        h["fp64_add_tops"] = sec["fp64_probe"]["fp64_add_tops"]
    i8 = {}
    for S in (6, 7, 8, 10):
        r = sec.get("dgemm_int8_8192_s%d" % S)
        if r:
            i8["s%d" % S] = [r["tflops_effective"], r["speedup_vs_plain"], r["int8_frac"],
                             float("%.3g" % r["err_over_binned_bound_max"])]
    h["dgemm_int8_8192"] = i8
    h["dgemm_int8_fields"] = "[effective TFLOP/s, x plain 8192, int8 frac, max err/dbbound]"
    h["dgemv_frac"] = {k[6:]: v["frac_of_copy_peak"] for k, v in sec.items()
                       if k.startswith("dgemv_")}
    b = sec.get("batched")
    if b:
        h["batched_ms"] = [b["ms"], b["segments_only_ms"], b["gemms_only_ms"],
                           b["spot_check_bit_identical"]]
    return h


def _event_time(torch, fn, reps, warm=1):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps * 1e-3


def int8_operands(rng, m, n):
    """mantissas uniform in [1, 2), exponents uniform in [-20, 20], random signs"""
    mant = rng.uniform(1.0, 2.0, (m, n))
    ex = rng.integers(-20, 21, (m, n))
    return np.ldexp(mant, ex) * rng.choice([-1.0, 1.0], (m, n))


def blas1_sweep(torch, rb):
    """Every BLAS1 reduction on HBM-resident inputs of 2^28 real elements (2^27 complex),
    fold 3: GB/s of algorithmic traffic and the fraction of the measured HBM copy peak."""
    peak, _ = peaks()
    g = torch.Generator(device="cuda").manual_seed(3)
    n = 1 << 28
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    xf, yf = x.float(), y.float()
    z = torch.zeros(2 * FOLD, dtype=torch.float64, device="cuda")
    zs = torch.zeros(2 * FOLD, dtype=torch.float32, device="cuda")
    zc = torch.zeros(4 * FOLD, dtype=torch.float64, device="cuda")
    zcf = torch.zeros(4 * FOLD, dtype=torch.float32, device="cuda")
    nc = n // 2   # complex elements over the same buffers
    cases = {
        "dsum": (8.0 * n, lambda: rb.call("binnedBLAS_dbdsum", FOLD, n, x, 1, z)),
        "ddot": (16.0 * n, lambda: rb.call("binnedBLAS_dbddot", FOLD, n, x, 1, y, 1, z)),
        "dnrm2_ssq": (8.0 * n, lambda: rb.call("binnedBLAS_dbdssq", FOLD, n, x, 1, 0.0, z)),
        "ssum": (4.0 * n, lambda: rb.call("binnedBLAS_sbssum", FOLD, n, xf, 1, zs)),
        "sdot": (8.0 * n, lambda: rb.call("binnedBLAS_sbsdot", FOLD, n, xf, 1, yf, 1, zs)),
        "zsum": (16.0 * nc, lambda: rb.call("binnedBLAS_zbzsum", FOLD, nc, x, 1, zc)),
        "zdotc": (32.0 * nc, lambda: rb.call("binnedBLAS_zbzdotc", FOLD, nc, x, 1, y, 1, zc)),
        "csum": (8.0 * (n // 2), lambda: rb.call("binnedBLAS_cbcsum", FOLD, n // 2, xf, 1, zcf)),
        "dasum": (8.0 * n, lambda: rb.call("binnedBLAS_dbdasum", FOLD, n, x, 1, z)),
        "sasum": (4.0 * n, lambda: rb.call("binnedBLAS_sbsasum", FOLD, n, xf, 1, zs)),
        "dzasum": (16.0 * nc, lambda: rb.call("binnedBLAS_dbzasum", FOLD, nc, x, 1, z)),
        "zdotu": (32.0 * nc, lambda: rb.call("binnedBLAS_zbzdotu", FOLD, nc, x, 1, y, 1, zc)),
        "cdotc": (16.0 * (n // 2), lambda: rb.call("binnedBLAS_cbcdotc", FOLD, n // 2, xf, 1, yf, 1, zcf)),
        "snrm2_ssq": (4.0 * n, lambda: rb.call("binnedBLAS_sbsssq", FOLD, n, xf, 1, 0.0, zs)),
        "dznrm2_ssq": (16.0 * nc, lambda: rb.call("binnedBLAS_dbzssq", FOLD, nc, x, 1, 0.0, z)),
    }
    out = {}
    for name, (byts, fn) in cases.items():
        t = _event_time(torch, fn, 10, warm=3)
        gbs = byts / t / 1e9
        out[name] = {"gbs": round(gbs, 1), "frac_of_copy_peak": round(gbs / peak, 3),
                     "us": round(t * 1e6, 1)}
    return out


def sweep_values(torch, dist, n, g):
    """Device vector of n FP64 values: uniform(-1,1), standard normal, log-uniform magnitude
    2^U(-300,300) with random sign, or ill-conditioned (x, -x) pairs plus n/16 entries of
    magnitude 1e-12, shuffled."""
    if dist == "uniform":
        return torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    if dist == "normal":
        return torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    if dist == "loguniform":
        e = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * 600 - 300
        sgn = torch.randint(0, 2, (n,), device="cuda", generator=g).double() * 2 - 1
        return torch.exp2(e) * sgn
    half = n // 2
    a = torch.rand(half, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    x = torch.cat([a, -a, torch.zeros(n - 2 * half, dtype=torch.float64, device="cuda")])
    k = n // 16
    idx = torch.randperm(n, device="cuda", generator=g)[:k]
    x[idx] = 1e-12
    return x[torch.randperm(n, device="cuda", generator=g)]


def blas1_full_sweep():
    """The BLAS1 sweep: dsum, ddot, dnrm2 (FP64), ssum, sdot (FP32), zsum, zdotc (complex128)
    at N = 2^10, 2^12, ..., 2^28 elements (complex: N/2 complex elements over the same bytes),
    folds 2, 3, 4, distributions uniform / normal / log-uniform / ill-conditioned; inputs
    resident in HBM; CUDA-event time per call over back-to-back calls (each call also reads its
    8-byte result back, as reproBLAS_r* do). Prints one JSON object: per routine, distribution
    and fold, {log2 N: [GB/s, us per call]}."""
    import torch
    import reproblas_b200 as rb
    g = torch.Generator(device="cuda").manual_seed(11)
    sizes = list(range(10, 29, 2))
    table = {}
    nmax = 1 << 28
    for dist in ("uniform", "normal", "loguniform", "illcond"):
        x = sweep_values(torch, dist, nmax, g)
        y = sweep_values(torch, dist, nmax, g)
        xf = x.float()
        yf = y.float()
        for fold in (2, 3, 4):
            cases = {
                "dsum": (8, lambda n: rb.call("reproBLAS_rdsum", fold, n, x, 1)),
                "ddot": (16, lambda n: rb.call("reproBLAS_rddot", fold, n, x, 1, y, 1)),
                "dnrm2": (8, lambda n: rb.call("reproBLAS_rdnrm2", fold, n, x, 1)),
                "ssum": (4, lambda n: rb.call("reproBLAS_rssum", fold, n, xf, 1)),
                "sdot": (8, lambda n: rb.call("reproBLAS_rsdot", fold, n, xf, 1, yf, 1)),
                "zsum": (8, lambda n: rb.call("reproBLAS_rzsum_sub", fold, n // 2, x, 1, out)),
                "zdotc": (16, lambda n: rb.call("reproBLAS_rzdotc_sub", fold, n // 2, x, 1, y, 1, out)),
            }
            out = torch.zeros(2, dtype=torch.float64, device="cuda")
            for name, (bpe, fn) in cases.items():
                row = {}
                for lg in sizes:
                    n = 1 << lg
                    reps = 20 if lg >= 24 else 200
                    t = _event_time(torch, lambda: fn(n), reps, warm=3)
                    row[lg] = [round(bpe * n / t / 1e9, 1), round(t * 1e6, 2)]
                table.setdefault(name, {}).setdefault(dist, {})[fold] = row
        del x, y, xf, yf
    print(json.dumps({"blas1_sweep": table, "unit": "[GB/s, us per call]",
                      "peak_gbs": peaks()[0], "peak_source": peaks()[1]}))


def batched_case(torch, rb, rng, profile_steps=0, total_log2=28):
    """Batched ragged configuration: 10,000 ddot segments with log-uniform lengths (drawn as
    floor(2^U(0,20)), then scaled so the total is ~2^28 elements, normal values) and 512
    dgemm instances with m, n, k uniform over {16..256}, uniform(-1,1), fold 3; autotuned
    schedule; one graph launch per step."""
    import ctypes
    nseg = 10000
    lens = np.floor(np.exp2(rng.uniform(0, 20, nseg)))
    lens = np.maximum(1, np.floor(lens * (2.0 ** total_log2 / lens.sum()))).astype(np.int32)
    offs = np.concatenate([[0], np.cumsum(lens.astype(np.int64))[:-1]]).astype(np.int64)
    total = int(lens.astype(np.int64).sum())
    X = torch.from_numpy(rng.standard_normal(total)).cuda()
    Y = torch.from_numpy(rng.standard_normal(total)).cuda()
    res = torch.zeros(nseg, dtype=torch.float64, device="cuda")
    ng = 512
    inst = (rb.DgemmInstance * ng)()
    keep = []
    flops = 0.0
    for g in range(ng):
        m, n, k = (int(v) for v in rng.integers(16, 257, 3))
        A = torch.from_numpy(rng.uniform(-1, 1, m * k)).cuda()
        B = torch.from_numpy(rng.uniform(-1, 1, k * n)).cuda()
        C = torch.from_numpy(rng.uniform(-1, 1, m * n)).cuda()
        keep += [A, B, C]
        d = inst[g]
        d.order, d.transa, d.transb = b"r", b"n", b"n"
        d.m, d.n, d.k, d.alpha, d.beta = m, n, k, 1.5, 0.5
        d.A, d.lda, d.B, d.ldb, d.C, d.ldc = A.data_ptr(), k, B.data_ptr(), n, C.data_ptr(), n
        flops += 2.0 * m * n * k
    plan = rb.lib.rb_batch_plan_create(3, nseg, offs.ctypes.data, lens.ctypes.data, X.data_ptr(),
                                       Y.data_ptr(), res.data_ptr(), None, ng, ctypes.addressof(inst))
    rb.check()
    if profile_steps:
        # profile case: the default schedule, no autotuning, no timing
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(profile_steps):
            rb.call("rb_batch_plan_run", plan, stream)
        torch.cuda.synchronize()
        rb.lib.rb_batch_plan_destroy(plan)
        return None
    t0 = time.perf_counter()
    rb.call("rb_batch_plan_autotune", plan, 3)
    tune_s = time.perf_counter() - t0
    info = [ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong(),
            ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
    rb.lib.rb_batch_plan_info(plan, *[ctypes.byref(v) for v in info])
    stream = torch.cuda.current_stream().cuda_stream
    t = _event_time(torch, lambda: rb.call("rb_batch_plan_run", plan, stream), 5, warm=2)
    # spot check: 64 segments equal the per-instance call
    srng = np.random.default_rng(5)
    got = res.cpu().numpy()
    same = True
    for i in srng.integers(0, nseg, 64):
        o, l = int(offs[i]), int(lens[i])
        same &= rb.call("reproBLAS_rddot", 3, l, X[o:], 1, Y[o:], 1) == got[i]
    rb.lib.rb_batch_plan_destroy(plan)
    # the two halves alone (same default schedule each): how much of them one launch overlaps
    parts = {}
    for name, ns, ngm in (("segments_only_ms", nseg, 0), ("gemms_only_ms", 0, ng)):
        p2 = rb.lib.rb_batch_plan_create(3, ns, offs.ctypes.data, lens.ctypes.data, X.data_ptr(),
                                         Y.data_ptr(), res.data_ptr(), None, ngm,
                                         ctypes.addressof(inst))
        rb.check()
        parts[name] = round(1e3 * _event_time(torch, lambda: rb.call("rb_batch_plan_run", p2, stream),
                                              5, warm=2), 3)
        rb.lib.rb_batch_plan_destroy(p2)
    return {"ms": round(t * 1e3, 3), **parts, "segments": nseg, "segment_elements": total,
            "dgemm_instances": ng, "reduction_gbs": round(16.0 * total / t / 1e9, 1),
            "gemm_tflops_if_alone": round(flops / t / 1e12, 3),
            "schedule": {"tile": [info[0].value, info[1].value], "chunk": info[2].value,
                         "small_max": info[3].value, "ctas_per_sm": info[4].value},
            "autotune": {"tried": info[5].value, "rejected": info[6].value, "seconds": round(tune_s, 2)},
            "spot_check_bit_identical": bool(same)}


def fp64_probe(torch, rb):
    """The FP64 rates that bound the plain binned dgemm, measured on this GPU: independent
    FP64 adds (the pipe's peak) and fl(a*b) products deposited into register-resident fold-3
    accumulators (rb_probe_launch kinds 0 and 1; CUDA-event time, best of 3)."""
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    res = {}
    for kind, iters, per in ((0, 1 << 16, 8), (1, 1 << 15, 4)):
        grid = sms * max(1, rb.lib.rb_probe_occupancy(kind))
        out = torch.empty(grid * 256, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        run = lambda: rb.call("rb_probe_launch", kind, iters, grid, out, stream)
        best = min(_event_time(torch, run, 1, warm=1) for _ in range(3))
        res[kind] = grid * 256.0 * iters * per / best
    return {"fp64_add_tops": round(res[0] / 1e12, 2),
            "binned_products_per_s_T": round(res[1] / 1e12, 3),
            "dgemm_ceiling_tflops": round(2 * res[1] / 1e12, 3),
            "note": "ceiling = 2 flops x the rate of fl(a*b) deposited into fold-3 accumulators "
                    "held in registers (no memory traffic); FP64 pipe peak for comparison"}


def secondary(args):
    """dgemm TFLOP/s, plain binned vs int8-sliced (the second half of the headline metric),
    and dgemv GB/s; rank 0 at N=1. Device-resident operands, CUDA-event timing."""
    import torch
    import reproblas_b200 as rb
    from _ffi import port, ptr
    out = {"blas1": blas1_sweep(torch, rb)}
    peak_bf16 = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak_bf16 = float(json.load(f)["bf16_tflops"])
    except Exception:
        peak_bf16 = 1590.0
    rng = np.random.default_rng(8192)
    # plain binned dgemm, the reference benchmark shape: M=N=K=2048, uniform(-1,1), alpha 1.5, beta 0.5
    n = 2048
    A = torch.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
    B = torch.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
    C0 = torch.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
    C = C0.clone()
    t = _event_time(torch, lambda: rb.call("reproBLAS_rdgemm", 3, "r", "n", "n", n, n, n, 1.5, A, n, B, n,
                                           0.5, C, n), 3)
    out["fp64_probe"] = fp64_probe(torch, rb)
    out["dgemm_plain_2048"] = {"tflops": round(2 * n ** 3 / t / 1e12, 4), "ms": round(t * 1e3, 3),
                               "bound": "fp64 pipe (binned deposit per product)",
                               "frac_of_deposit_ceiling": round(2 * n ** 3 / t / 1e12 /
                                                                out["fp64_probe"]["dgemm_ceiling_tflops"], 3)}
    del A, B, C, C0
    # 8192^3: plain binned vs int8-sliced on the int8 configuration's data
    n = 8192
    Ah = int8_operands(rng, n, n)
    Bh = int8_operands(rng, n, n)
    Ch = rng.uniform(-1, 1, (n, n))
    A = torch.from_numpy(Ah).cuda(); B = torch.from_numpy(Bh).cuda()
    C = torch.from_numpy(Ch).cuda()
    t_plain = _event_time(torch, lambda: rb.call("reproBLAS_rdgemm", 3, "r", "n", "n", n, n, n, 1.5, A, n,
                                                 B, n, 0.5, C, n), 1, warm=1)
    out["dgemm_plain_8192"] = {"tflops": round(2 * n ** 3 / t_plain / 1e12, 4),
                               "ms": round(t_plain * 1e3, 2)}
    for S in (6, 7, 8, 10):
        C.copy_(torch.from_numpy(Ch))
        t8 = _event_time(torch, lambda: rb.call("rb_dgemm_int8", 3, "r", "n", "n", n, n, n, 1.5, A, n, B,
                                                n, 0.5, C, n, S), 3)
        pairs = S * (S + 1) // 2
        tops = 2.0 * pairs * n ** 3 / t8 / 1e12
        rec = {"tflops_effective": round(2 * n ** 3 / t8 / 1e12, 3), "ms": round(t8 * 1e3, 3),
               "slices": S, "digit_pairs": pairs, "int8_tops_issued": round(tops, 1),
               "int8_peak_tops": round(2 * peak_bf16, 1),
               "int8_frac": round(tops / (2 * peak_bf16), 4),
               "speedup_vs_plain": round(t_plain / t8, 2)}
        # error vs the exact host oracle on 4096 sampled entries, beside binned_dbbound
        C.copy_(torch.from_numpy(Ch))
        rb.call("rb_dgemm_int8", 3, "r", "n", "n", n, n, n, 1.5, A, n, B, n, 0.5, C, n, S)
        got = C.cpu().numpy()
        P = port()
        srng = np.random.default_rng(S)
        errs, ratios = [], []
        for _ in range(4096):
            i, j = int(srng.integers(0, n)), int(srng.integers(0, n))
            a = np.ascontiguousarray(np.concatenate([Ah[i, :] * 1.5, [Ch[i, j] * 0.5]]))
            b = np.ascontiguousarray(np.concatenate([Bh[:, j], [1.0]]))
            ex = P.exact_dot(n + 1, ptr(a), 1, ptr(b), 1)
            err = abs(got[i, j] - ex)
            bound = P.dbbound(3, n + 1, float(np.max(np.abs(a * b))), ex)
            errs.append(err / max(abs(ex), 1e-300))
            ratios.append(err / bound)
        rec["rel_err_max"] = float(np.max(errs))
        rec["rel_err_mean"] = float(np.mean(errs))
        rec["err_over_binned_bound_max"] = float(np.max(ratios))
        rec["err_over_binned_bound_mean"] = float(np.mean(ratios))
        out["dgemm_int8_8192_s%d" % S] = rec
    del A, B, C
    out["batched"] = batched_case(torch, rb, rng)
    # dgemv, NoTrans (row reduction) and Trans (column reduction), row-major A, alpha 1.5,
    # beta 0.5, fold 3: the three 128 MiB shapes of the reference's gemv benchmark and
    # 16384^2 (2 GiB). "us" is CUDA-event time per call over back-to-back calls, "host_us"
    # the host time of one call (the call returns after enqueueing, so us ~ host_us would
    # mean host-bound).
    for (m, n) in ((4096, 4096), (16384, 1024), (1024, 16384), (16384, 16384)):
        A = torch.from_numpy(rng.uniform(-1, 1, (m, n))).cuda()
        for ta in "nt":
            lx, ly = (n, m) if ta == "n" else (m, n)
            x = torch.from_numpy(rng.uniform(-1, 1, lx)).cuda()
            y = torch.from_numpy(rng.uniform(-1, 1, ly)).cuda()
            call = lambda: rb.call("reproBLAS_rdgemv", 3, "r", ta, m, n, 1.5, A, n, x, 1, 0.5, y, 1)
            reps = 5 if m * n > 2 ** 26 else 20
            t = _event_time(torch, call, reps, warm=3)
            torch.cuda.synchronize()
            h0 = time.perf_counter()
            call()
            h1 = time.perf_counter()
            torch.cuda.synchronize()
            byts = 8.0 * m * n + 8.0 * lx + 16.0 * ly
            out["dgemv_%dx%d_%s" % (m, n, ta)] = {
                "gbs": round(byts / t / 1e9, 1), "us": round(t * 1e6, 2),
                "host_us": round((h1 - h0) * 1e6, 1),
                "frac_of_copy_peak": round(byts / t / 1e9 / peaks()[0], 3)}
            del x, y
        del A
    out.update(xblas23_cases(torch, rb, rng))
    return out


def xblas23_cases(torch, rb, rng):
    """FP32 real / FP64 complex / FP32 complex gemv (NoTrans and ConjTrans, 128 MiB and 1 GiB
    matrices) and gemm (M = N = K = 1024), row-major, fold 3, alpha 1.5 (complex 1.5 - 0.25i),
    beta 0.5, device-resident operands. gemv bytes: A + x + y read + y written; gemm work in
    real flops (complex: 8 per multiply-add) and binned deposits (complex: 4 per multiply-add)."""
    out = {}
    real = {"s": np.float32, "z": np.float64, "c": np.float32}
    shapes = {"s": ((8192, 4096), (16384, 16384)), "z": ((4096, 2048), (8192, 8192)),
              "c": ((4096, 4096), (8192, 16384))}
    for t in "szc":
        nc = 1 if t == "s" else 2
        es = np.dtype(real[t]).itemsize * nc
        al = 1.5 if t == "s" else np.array([1.5, -0.25], real[t])
        be = 0.5 if t == "s" else np.array([0.5, 0.0], real[t])
        for (m, n) in shapes[t]:
            A = torch.from_numpy(rng.uniform(-1, 1, m * n * nc).astype(real[t])).cuda()
            for ta in ("n", "c" if t != "s" else "t"):
                lx, ly = (n, m) if ta == "n" else (m, n)
                x = torch.from_numpy(rng.uniform(-1, 1, lx * nc).astype(real[t])).cuda()
                y = torch.from_numpy(rng.uniform(-1, 1, ly * nc).astype(real[t])).cuda()
                call = lambda: rb.call("reproBLAS_r%sgemv" % t, 3, "r", ta, m, n, al, A, n, x, 1, be, y, 1)
                t_s = _event_time(torch, call, 5 if m * n * es > 2 ** 28 else 20, warm=3)
                byts = float(es) * (m * n + lx + 2 * ly)
                out["%sgemv_%dx%d_%s" % (t, m, n, ta)] = {
                    "gbs": round(byts / t_s / 1e9, 1), "us": round(t_s * 1e6, 2),
                    "frac_of_copy_peak": round(byts / t_s / 1e9 / peaks()[0], 3)}
                del x, y
            del A
        k = 1024
        A = torch.from_numpy(rng.uniform(-1, 1, k * k * nc).astype(real[t])).cuda()
        B = torch.from_numpy(rng.uniform(-1, 1, k * k * nc).astype(real[t])).cuda()
        C = torch.from_numpy(rng.uniform(-1, 1, k * k * nc).astype(real[t])).cuda()
        t_s = _event_time(torch, lambda: rb.call("reproBLAS_r%sgemm" % t, 3, "r", "n", "n", k, k, k, al, A, k,
                                                 B, k, be, C, k), 3, warm=1)
        flops = (2.0 if t == "s" else 8.0) * k ** 3
        out["%sgemm_1024" % t] = {"gflops": round(flops / t_s / 1e9, 1), "ms": round(t_s * 1e3, 3),
                                  "gdeposits_per_s": round(k ** 3 * nc * nc / t_s / 1e9, 1)}
        del A, B, C
    return out


def profile_case(args):
    """A small case of one kernel for ncu captures (prints nothing but a short note)."""
    import torch
    import reproblas_b200 as rb
    rng = np.random.default_rng(1)
    n = args.profile_n
    if args.profile_kernel in ("gemv_n", "gemv_t"):
        m = args.profile_m or n
        ta = args.profile_kernel[-1]
        A = torch.from_numpy(rng.uniform(-1, 1, (m, n))).cuda()
        x = torch.from_numpy(rng.uniform(-1, 1, n if ta == "n" else m)).cuda()
        y = torch.from_numpy(rng.uniform(-1, 1, m if ta == "n" else n)).cuda()
        for _ in range(args.warmup + args.steps):
            rb.call("reproBLAS_rdgemv", 3, "r", ta, m, n, 1.5, A, n, x, 1, 0.5, y, 1)
        torch.cuda.synchronize()
        print("profile case done: %s m=%d n=%d" % (args.profile_kernel, m, n))
        return
    if args.profile_kernel[0] in "szc" and args.profile_kernel[1:4] == "gem":
        # FP32 real / complex gemv (m x n, row-major) or gemm (n^3), fold 3, uniform(-1, 1)
        t, kind = args.profile_kernel[0], args.profile_kernel[1:5]
        nc = 1 if t == "s" else 2
        real = np.float64 if t == "z" else np.float32
        al = 1.5 if t == "s" else np.array([1.5, -0.25], real)
        be = 0.5 if t == "s" else np.array([0.5, 0.0], real)
        m = args.profile_m or n
        if kind == "gemv":
            ta = args.profile_kernel[-1]
            A = torch.from_numpy(rng.uniform(-1, 1, m * n * nc).astype(real)).cuda()
            x = torch.from_numpy(rng.uniform(-1, 1, (n if ta == "n" else m) * nc).astype(real)).cuda()
            y = torch.from_numpy(rng.uniform(-1, 1, (m if ta == "n" else n) * nc).astype(real)).cuda()
            for _ in range(args.warmup + args.steps):
                rb.call("reproBLAS_r%sgemv" % t, 3, "r", ta, m, n, al, A, n, x, 1, be, y, 1)
        else:
            A, B, C = (torch.from_numpy(rng.uniform(-1, 1, n * n * nc).astype(real)).cuda()
                       for _ in range(3))
            for _ in range(args.warmup + args.steps):
                rb.call("reproBLAS_r%sgemm" % t, 3, "r", "n", "n", n, n, n, al, A, n, B, n, be, C, n)
        torch.cuda.synchronize()
        print("profile case done: %s m=%d n=%d" % (args.profile_kernel, m, n))
        return
    if args.profile_kernel == "batched":
        # a quarter of the benchmark's segment elements (2^26), the same 512 dgemm instances
        batched_case(torch, rb, rng, profile_steps=args.warmup + args.steps, total_log2=26)
        print("profile case done: batched")
        return
    if args.profile_kernel in ("zdotc", "zsum", "csum", "dnrm2"):
        # n elements (complex for the z/c routines), uniform(-1, 1), fold 3
        k = args.profile_kernel
        comps = 1 if k == "dnrm2" else 2
        dt = torch.float32 if k == "csum" else torch.float64
        X = torch.from_numpy(rng.uniform(-1, 1, comps * n)).to(dt).cuda()
        Y = torch.from_numpy(rng.uniform(-1, 1, comps * n)).to(dt).cuda()
        out = torch.zeros(2, dtype=dt, device="cuda")
        for _ in range(args.warmup + args.steps):
            if k == "zdotc":
                rb.call("reproBLAS_rzdotc_sub", 3, n, X, 1, Y, 1, out)
            elif k == "zsum":
                rb.call("reproBLAS_rzsum_sub", 3, n, X, 1, out)
            elif k == "csum":
                rb.call("reproBLAS_rcsum_sub", 3, n, X, 1, out)
            else:
                rb.call("reproBLAS_rdnrm2", 3, n, X, 1)
        torch.cuda.synchronize()
        print("profile case done: %s n=%d" % (k, n))
        return
    A = torch.from_numpy(int8_operands(rng, n, n)).cuda()
    B = torch.from_numpy(int8_operands(rng, n, n)).cuda()
    C = torch.from_numpy(rng.uniform(-1, 1, (n, n))).cuda()
    for _ in range(args.warmup + args.steps):
        if args.profile_kernel == "int8":
            rb.call("rb_dgemm_int8", 3, "r", "n", "n", n, n, n, 1.5, A, n, B, n, 0.5, C, n,
                    args.profile_slices)
        else:
            rb.call("reproBLAS_rdgemm", 3, "r", "n", "n", n, n, n, 1.5, A, n, B, n, 0.5, C, n)
    torch.cuda.synchronize()
    print("profile case done: %s n=%d" % (args.profile_kernel, n))


def main():
    args = parse()
    if args.profile_kernel:
        profile_case(args)
        return
    if args.sweep:
        blas1_full_sweep()
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank)
    else:
        ours_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
