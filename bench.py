"""Benchmark of the big-integer multiply path (one JSON line on rank 0).

Default workload (configuration 2): one plain 2^28-bit x 2^28-bit product
(2^23 u32 words each, uniform random with the top bit set, seeded), 32-bit
coefficients, n = 2^24, two 58-bit primes (64-bit prime path); the library's
plan for it runs 64-bit coefficients over three primes.  A "step" is
one full product.  Metric: products/s (whole job), with the per-stage times,
the HBM roofline of the dominant kernel and the product-level algorithmic
byte model (12*K*n*w + in + out) beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config 1|2|2sq|4|3|5]

Configurations: 2 (default), 2sq (squaring), 1 (2^20-bit, 32-bit path), 4
(2^33-bit, n = 2^29, three passes), 3 (4096 batched products of uneven
sizes, against the plain path looped per product), 5 (serving: open-loop
Poisson arrivals, p50/p99 latency); prof and 3prof are smaller cases of the
same kernels for ncu captures.

Multi-GPU: products are independent, so N ranks run N replicas (no
collective on the data path, "scaling": "weak"); the timed region is
bracketed by a barrier and the max over ranks is reported.

--impl reference times the CPU restatement of the reference's algorithm
(oracle/, the reference has no CPU multiply of its own and its GPU NTT
library is absent) on this host's cores, on the same configuration.
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

L2_BYTES = 126 * 1024 * 1024
FALLBACK_HBM_GBS = 6650.0

# Plain single-product configurations come from the table the parity tests
# also read (birdwing_b200.workloads.PLAIN): name -> (words_a, words_b, path,
# K, square, description) of the reference's algorithm, which the oracle, the
# CPU baseline and --impl reference run; the library's plan is built from the
# same table's `plan` entry (plain_plan_args) and the JSON line reports what
# it resolved to (coeff_bits, num_primes, log_n).
from birdwing_b200.workloads import PLAIN, algorithm_of, plain_plan_args  # noqa: E402

CONFIGS = {name: (w["words_a"], w["words_b"], w["ref"][0], w["ref"][1], w["square"], w["desc"])
           for name, w in PLAIN.items()}


def ref_algorithm(cfg):
    """The reference's algorithm for a plain configuration, in words."""
    la, lb, path, K, square, _ = CONFIGS[cfg]
    cpw = 2 if path == 32 else 1
    log_n = max(4, ((la + (la if square else lb)) * cpw - 2).bit_length())
    return (f"reference algorithm: {32 // cpw}-bit coefficients, n=2^{log_n}, {K} x "
            f"{58 if path == 64 else 30}-bit primes (CPU restatement)")


# batched configurations: (products, seed, K, description)
BATCH_CONFIGS = {
    "3": (4096, 3, 2,
          "batched uneven sizes: 4096 products, operands 2^12..2^20 bits log-uniform, second "
          "operand 1/8x..1x, half on the 32-bit path (16-bit coefficients), half on the "
          "64-bit path (32-bit coefficients), 2 primes each"),
    # the same mix at 1/8 of the products, for ncu captures
    "3prof": (512, 3, 2, "batched uneven sizes, 512 products of the same mix"),
}

# serving configurations: (distinct requests in the pool, seed, K, description)
SERVE_CONFIGS = {
    "5": (1024, 5, 2,
          "serving: open-loop Poisson arrivals, operands 2^10..2^24 bits log-uniform, 20% "
          "squarings, second operand 1/8x..1x, prime path chosen per request (automatic), "
          "2 primes, 120 GiB admission budget"),
}


def parse():
    return parse_args_list(None)


def parse_args_list(argv):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="2",
                    choices=sorted(CONFIGS) + sorted(BATCH_CONFIGS) + sorted(SERVE_CONFIGS) + ["intpeak"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--autotune", action="store_true",
                    help="batched configurations: tune each bucket's kernel form first")
    ap.add_argument("--no-plain", action="store_true",
                    help="batched/serving configurations: skip the plain per-product path")
    ap.add_argument("--duration", type=float, default=10.0,
                    help="serving: seconds of arrivals per swept rate")
    ap.add_argument("--rate-fracs", default="0.3,0.45,0.6,0.75",
                    help="serving: arrival rates as fractions of the closed-loop capacity")
    ap.add_argument("--log-cols", type=int, default=0,
                    help="4-step split override (BW_PLAN_LOG_COLS), 0 = automatic")
    ap.add_argument("--plan-flags", type=lambda s: int(s, 0), default=0,
                    help="extra bw_plan_create flags (tuning switches)")
    ap.add_argument("--persistent", action="store_true",
                    help="batched configurations: small buckets as one persistent kernel per "
                         "path over a device work queue (BW_BATCH_PERSISTENT)")
    ap.add_argument("--no-sub", action="store_true",
                    help="plain configuration 2: skip the batched and serving sub-records")
    return ap.parse_args(argv)


def operands(cfg, rank):
    from oracle import mt64
    la, lb, path, K, square, _ = CONFIGS[cfg]
    sa, sb = PLAIN[cfg]["seeds"]
    a = mt64.random_words_top_fast(la, sa + 1000 * rank)
    b = a if square else mt64.random_words_top_fast(lb, sb + 1000 * rank)
    return a, b


def model_bytes(la, lb, n, K, w, square):
    """Per-kernel split of the fixed algorithmic byte model
    12*K*n*w + in + out (9*K*n*w + in + out when squaring)."""
    knw = K * n * w
    ops = 1 if square else 2
    fwd = 4 * (la + (0 if square else lb)) + ops * knw          # FWD pass 1 (A, B)
    row = ops * 2 * knw + 3 * knw                               # FWD pass 2 + INV pass 1
    inv = 2 * knw                                               # INV pass 2
    carry = knw + 4 * (la + lb)                                 # Garner + carry
    return {"fwd_ms": fwd, "mul_ms": row, "intt_ms": inv, "crt_carry_ms": carry}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def load_traffic(cfg, kernel):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)[cfg][kernel]
    except Exception:
        return None


def reduce_over_ranks(values, ops):
    """All-reduce one float per entry across the job's ranks: "max" for times
    (the slowest rank bounds the job), "sum" for counts.  A no-op on a single
    process.  Runs on the GPU under NCCL and on the CPU under gloo."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    out = []
    for v, op in zip(values, ops):
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        out.append(float(t.item()))
    return out


def job_throughput(units_per_rank, world, rank_ms):
    """Whole-job units/s: every rank processed units_per_rank units and the
    job took the slowest rank's time (ms, already reduced with max)."""
    return world * units_per_rank / (rank_ms * 1e-3)


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region.  NVML (the library nvidia-smi reads) is polled every 2 ms from a
    thread, so that even a timed region of a few tens of milliseconds holds
    samples; `region(t0, t1)` marks the timed region (time.perf_counter
    values) and the summary covers the samples inside it.  Without NVML,
    nvidia-smi is sampled every 100 ms instead."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index, period_s=0.002):
        self.gpu = gpu_index
        self.period = period_s
        self.samples = []           # (t, sm_mhz, sm_max_mhz, set of reasons)
        self.window = None
        self.proc = None
        self.nvml = None
        self.lines = []

    def start(self):
        try:
            import pynvml as N
            N.nvmlInit()
            self.nvml = N
            self.h = N.nvmlDeviceGetHandleByIndex(self.gpu)
            self.smax = N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM)
            self.bits = {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
                         "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
                         "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
                         "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap}
            self.stop_flag = False
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _poll(self):
        N = self.nvml
        while not self.stop_flag:
            try:
                sm = N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM)
                r = N.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((time.perf_counter(), float(sm), float(self.smax),
                                     {k for k, bit in self.bits.items() if r & bit}))
            except Exception:
                pass
            time.sleep(self.period)

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm, smax = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            reasons = {nm for nm, v in zip(self.REASONS, parts[5:9]) if v.lower() == "active"}
            self.samples.append((time.perf_counter(), sm, smax, reasons))

    def region(self, t0, t1):
        self.window = (t0, t1)

    def stop(self):
        if self.nvml is not None:
            self.stop_flag = True
            self.t.join(timeout=2)
            source = "NVML every 2 ms"
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)
            source = "nvidia-smi every 100 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sel = self.samples
        if self.window:
            t0, t1 = self.window
            inside = [x for x in sel if t0 <= x[0] <= t1]
            sel = inside or sel
        sm = [x[1] for x in sel]
        reasons = set().union(*[x[3] for x in sel]) if sel else set()
        out = {"sm_mhz": statistics.median(sm) if sm else None,
               "sm_max_mhz": max(x[2] for x in sel) if sel else None,
               "samples": len(sel), "reasons": sorted(reasons), "source": source}
        if self.window:
            out["region_ms"] = 1000.0 * (self.window[1] - self.window[0])
            out["samples_in_region"] = len([x for x in self.samples
                                            if self.window[0] <= x[0] <= self.window[1]])
        return out


def residue_check(a, b, got, count=3, seed=61):
    """Product check without a full multiprecision multiply: the result's
    residues mod 2^64 and mod `count` random 61-bit probable primes."""
    def as_int(w):
        return int.from_bytes(np.ascontiguousarray(w).view(np.uint8).tobytes(), "little")
    A, B, C = as_int(a), as_int(b), as_int(got)
    rng = np.random.default_rng(seed)
    mods = [1 << 64]
    while len(mods) < count + 1:
        m = int(rng.integers(1 << 60, 1 << 61)) | 1
        if pow(3, m - 1, m) == 1:
            mods.append(m)
    return all(C % m == (A % m) * (B % m) % m for m in mods)


# configurations too large for a full CPU product inside the baseline budget:
# the oracle runs a smaller product of the same path and primes, and its time
# is scaled by n log n (the transforms dominate)
CPU_SAMPLE_WORDS = {"4": 1 << 22}


def cpu_baseline(cfg, budget_s=20.0):
    """The oracle (CPU restatement of the reference's algorithm) with all host
    threads on the same operands: full products until the budget is spent
    (at least one).  GMP mpz_mul (single thread) is reported beside it."""
    from oracle import gmp_ref, oracle
    la, lb, path, K, square, _ = CONFIGS[cfg]
    if cfg in CPU_SAMPLE_WORDS:
        return cpu_baseline_scaled(cfg, CPU_SAMPLE_WORDS[cfg], budget_s)
    a, b = operands(cfg, 0)
    cores = os.cpu_count() or 1
    oracle.lib.oracle_set_threads(cores)
    n_done, t0 = 0, time.perf_counter()
    while True:
        oracle.multiply(a, b, path, K)
        n_done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    g = gmp_ref.time_mul(a, b, 1)
    return {"value": n_done / dt, "unit": "products/s", "cores": cores, "kind": "port",
            "sample": f"{n_done} full product(s) of the workload, oracle/bw_oracle.c on "
                      f"{cores} threads, {dt:.1f} s",
            "gmp": {"value": 1.0 / g, "unit": "products/s", "cores": 1,
                    "impl": f"GMP {gmp_ref.version} mpz_mul, single thread"}}


def cpu_baseline_scaled(cfg, words, budget_s):
    from oracle import gmp_ref, mt64, oracle
    la, lb, path, K, square, _ = CONFIGS[cfg]
    a = mt64.random_words_top_fast(words, 1234)
    b = a if square else mt64.random_words_top_fast(words, 5678)
    cores = os.cpu_count() or 1
    oracle.lib.oracle_set_threads(cores)
    n_done, t0 = 0, time.perf_counter()
    while True:
        oracle.multiply(a, b, path, K)
        n_done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = (time.perf_counter() - t0) / n_done
    log_s = max(4, (2 * words - 2).bit_length())
    log_f = max(4, (la + lb - 2).bit_length())
    scale = ((1 << log_f) * log_f) / ((1 << log_s) * log_s)
    g = gmp_ref.time_mul(a, b, 1) * scale
    return {"value": 1.0 / (dt * scale), "unit": "products/s", "cores": cores, "kind": "port",
            "sample": f"{n_done} product(s) of {words} x {words} words (n = 2^{log_s}) with the "
                      f"workload's path and primes, oracle/bw_oracle.c on {cores} threads, "
                      f"{dt:.2f} s each, scaled by n log n to n = 2^{log_f} (x{scale:.1f})",
            "gmp": {"value": 1.0 / g, "unit": "products/s", "cores": 1,
                    "impl": f"GMP {gmp_ref.version} mpz_mul, single thread, same sample "
                            f"and scaling"}}


def run_reference(args):
    """--impl reference: the oracle port on the host cores, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    la, lb, path, K, square, desc = CONFIGS[args.config]
    if args.config in CPU_SAMPLE_WORDS:
        cb = cpu_baseline_scaled(args.config, CPU_SAMPLE_WORDS[args.config], 60.0)
        v = cb["value"]
        print(json.dumps({
            "impl": "reference", "metric": "products/s", "value": v, "unit": "products/s",
            "n_gpus": args.gpus, "steps": 1, "warmup": 0, "ms_per_step": 1000.0 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "config": {"workload": f"config {args.config}: {desc}",
                                            "algorithm": ref_algorithm(args.config),
                                            "words_a": la, "words_b": lb, "path": path,
                                            "num_primes": K},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "products/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}))
        return
    a, b = operands(args.config, 0)
    cores = os.cpu_count() or 1
    oracle.lib.oracle_set_threads(cores)
    t0 = time.perf_counter()
    oracle.multiply(a, b, path, K)
    t_one = time.perf_counter() - t0
    # bounded: at most ~150 s of timed work whatever --steps asks for
    steps = max(1, min(args.steps, int(150.0 / max(t_one, 1e-3))))
    warm = min(args.warmup, 1)
    for _ in range(warm):
        oracle.multiply(a, b, path, K)
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.multiply(a, b, path, K)
    dt = time.perf_counter() - t0
    v = steps / dt
    line = {
        "impl": "reference", "metric": "products/s", "value": v, "unit": "products/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": 1000 * dt / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": {"workload": f"config {args.config}: {desc}",
                                        "algorithm": ref_algorithm(args.config),
                                        "words_a": la, "words_b": lb, "path": path,
                                        "num_primes": K},
        "cpu_baseline": {"value": v, "unit": "products/s", "cores": cores, "kind": "port",
                         "sample": f"{steps} full products (requested {args.steps}), "
                                   f"oracle/bw_oracle.c on {cores} threads"},
        "e2e": {"value": v, "unit": "products/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference's GPU pipeline needs the absent GPU-NTT library; this is the "
                "CPU restatement of its algorithm (radix-2 NTT, Garner, carry)",
    }
    print(json.dumps(line))


def batch_items(cfg, rank):
    from birdwing_b200 import workloads
    count, seed, K, _ = BATCH_CONFIGS[cfg]
    return workloads.batch_mix(count, seed=seed + 100 * rank), K


def plain_launches(path, la, lb):
    """Kernels one plain product launches: the three transform passes, then
    the boundary pre-pass, the words pass and the carry fix when the output
    spans more than one 2048-word tile (the words pass alone otherwise)."""
    cpw = 2 if path == 32 else 1
    log_n = max(4, ((la + lb) * cpw - 2).bit_length())
    words = max((1 << log_n) // cpw, la + lb)
    return 3 + (3 if words > 2048 else 1)


def batch_model_bytes(items, K, small_max=None):
    """Algorithmic HBM bytes of a batch: per product the plain path's model
    (12*K*n*w + in + out) for 4-step products, and in + out + 2*K*n*w (one
    residue write and read) for products run one CTA each."""
    small_max = small_max or {64: 12, 32: 12}   # the library's default forms
    total = 0
    for p, a, b in items:
        cpw = 2 if p == 32 else 1
        w = 8 if p == 64 else 4
        log_n = max(4, ((len(a) + len(b)) * cpw - 2).bit_length())
        knw = K * (1 << log_n) * w
        io = 4 * (len(a) + len(b)) * 2
        total += io + (2 * knw if log_n <= small_max[p] else 12 * knw)
    return total


def cpu_baseline_items(items, K, budget_s=20.0):
    """The oracle on all host threads over the batch's products in order until
    the budget is spent; GMP mpz_mul (one thread) over all of them."""
    from oracle import gmp_ref, oracle
    cores = os.cpu_count() or 1
    oracle.lib.oracle_set_threads(cores)
    n_done, t0 = 0, time.perf_counter()
    for p, a, b in items:
        oracle.multiply(a, b, p, K)
        n_done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    g = sum(gmp_ref.time_mul(a, b, 1) for _, a, b in items)
    return {"value": n_done / dt, "unit": "products/s", "cores": cores, "kind": "port",
            "sample": f"first {n_done} of {len(items)} products of the mix, oracle/bw_oracle.c "
                      f"on {cores} threads, {dt:.1f} s",
            "gmp": {"value": len(items) / g, "unit": "products/s", "cores": 1,
                    "impl": f"GMP {gmp_ref.version} mpz_mul, single thread, all products"}}


def bench_batch(args):
    """Batched configuration: the whole mix is one step (one graph launch)."""
    import torch
    import torch.distributed as dist

    import birdwing_b200 as bw
    from birdwing_b200 import _lib as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_over_ranks([x], ["max"])[0]

    items, K = batch_items(args.config, rank)
    count, _, _, desc = BATCH_CONFIGS[args.config]
    stream = torch.cuda.Stream()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    # operands in pinned host memory (the batch copies them in and out)
    pinned = []
    for p, a, b in items:
        ha = torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32)
        hb = torch.from_numpy(b.view(np.int32)).pin_memory().numpy().view(np.uint32)
        pinned.append((p, ha, hb))
    bt = bw.Batch(num_primes=K, stream=stream.cuda_stream, persistent=args.persistent)
    outs = [bt.add(a, b, path=p) for p, a, b in pinned]
    if args.autotune:
        bt.autotune(reps=3)
    bt.run()                                   # layout, graph, upload, compute, download
    info = bt.info()
    if rank == 0:
        from oracle import gmp_ref
        ok = all(bool((o == gmp_ref.mul(a, b)).all()) for o, (_, a, b) in zip(outs, items))
    else:
        ok = True
    for _ in range(max(3, args.warmup)):
        bt.run(L.BW_BATCH_COMPUTE)

    sampler = ClockSampler(local)
    per_step = []
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.3)
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(i)                     # evict L2 between steps
        t = bt.run(L.BW_BATCH_COMPUTE, timing=True)
        per_step.append(t["mul_ms"])
    torch.cuda.synchronize()
    clocks = sampler.stop()
    barrier()
    total_ms = max_over_ranks(sum(per_step))

    # end to end through the public API: host operands in, host results out
    barrier()
    e2e_ms = []
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        bt.run()
        e2e_ms.append(1000 * (time.perf_counter() - t0))
    e2e_total = max_over_ranks(sum(e2e_ms))

    # the plain path looped product by product on the same GPU: one plan and
    # context per size (built before timing), all on one stream
    plain = None
    if not args.no_plain:
        plans, ctxs, bufs = [], [], []
        for p, a, b in items:
            pl = bw.Plan(len(a), len(b), p, K)
            plans.append(pl)
            ctxs.append(bw.Context(pl, stream=stream.cuda_stream))
            da = torch.from_numpy(a.view(np.int32)).cuda()
            db = torch.from_numpy(b.view(np.int32)).cuda()
            dc = torch.empty(len(a) + len(b), dtype=torch.int32, device="cuda")
            bufs.append((da, db, dc))

        def loop():
            for c, (da, db, dc) in zip(ctxs, bufs):
                c.multiply_device(da.data_ptr(), da.numel(), db.data_ptr(), db.numel(),
                                  dc.data_ptr(), dc.numel())

        loop()
        ctxs[0].sync()
        if rank == 0:
            from oracle import gmp_ref
            for j in range(0, len(items), 97):
                _, a, b = items[j]
                assert (bufs[j][2].cpu().numpy().view(np.uint32) == gmp_ref.mul(a, b)).all()
        reps = max(1, min(args.steps, 5))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            flush.fill_(0)
            e0.record(stream)
        for _ in range(reps):
            loop()
        with torch.cuda.stream(stream):
            e1.record(stream)
        torch.cuda.synchronize()
        for c in ctxs:
            c.sync()
        plain_ms = max_over_ranks(e0.elapsed_time(e1) / reps)
        plain = {"value": world * count / (plain_ms * 1e-3), "unit": "products/s",
                 "ms_per_step": plain_ms,
                 "gpu_launches_per_step": sum(plain_launches(p, len(a), len(b))
                                              for p, a, b in items),
                 "how": "bw_multiply (device pointers) per product, one plan+context per "
                        "product size built beforehand, one stream"}
        for c in ctxs:
            c.close()
        for pl in plans:
            pl.close()

    if rank == 0:
        ms = total_ms / args.steps
        peak, peak_kind = load_peaks()
        mb = batch_model_bytes(items, K)
        achieved = mb / (ms * 1e-3) / 1e9
        launches = info["kernel_nodes"]
        h2d = sum(4 * (len(a) + len(b)) for _, a, b in items)
        d2h = sum(4 * (len(a) + len(b)) for _, a, b in items) + 4
        line = {
            "metric": "products/s", "value": job_throughput(count * args.steps, world, total_ms),
            "unit": "products/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64/u32", "data": "synthetic",
            "config": {"workload": f"config {args.config}: {desc}", "products": count,
                       "num_primes": K, "buckets": info["buckets"],
                       "small_buckets": info["small_buckets"],
                       "graph_nodes": info["graph_nodes"],
                       "device_bytes": info["device_bytes"], "autotuned": bool(args.autotune),
                       "small_form": "persistent queue kernel per path" if args.persistent
                                     else "graph of per-bucket grids",
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas x{world}"},
            "correct_vs_gmp": ok,
            "roofline": {"bound": "hbm", "kernel": "batch graph (all buckets, one launch)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": load_traffic(args.config, "batch_graph"),
                         "algorithmic_bytes": mb},
            "plain_loop": plain,
            "batched_over_plain": (world * count * args.steps / (total_ms * 1e-3)) /
                                  plain["value"] if plain else None,
            "e2e": {"value": world * count * args.e2e_steps / (e2e_total * 1e-3),
                    "unit": "products/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches * args.steps,
            "clocks": clocks,
            "tune_table": bw.tune_table() if args.autotune else None,
        }
        if not args.no_cpu_baseline and world == 1:   # the CPU baseline runs at N = 1 only
            line["cpu_baseline"] = cpu_baseline_items(items, K)
        print(json.dumps(line))
    bt.close()
    if world > 1:
        dist.destroy_process_group()


def run_reference_batch(args):
    """--impl reference on a batched configuration: the oracle over the mix's
    products in order (a bounded sample), on all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    items, K = batch_items(args.config, 0)
    count, _, _, desc = BATCH_CONFIGS[args.config]
    cores = os.cpu_count() or 1
    oracle.lib.oracle_set_threads(cores)
    for p, a, b in items[: min(args.warmup, 3)]:
        oracle.multiply(a, b, p, K)
    budget = 150.0
    n_done, t0 = 0, time.perf_counter()
    for p, a, b in items:
        oracle.multiply(a, b, p, K)
        n_done += 1
        if time.perf_counter() - t0 >= budget:
            break
    dt = time.perf_counter() - t0
    v = n_done / dt
    line = {
        "impl": "reference", "metric": "products/s", "value": v, "unit": "products/s",
        "n_gpus": args.gpus, "steps": 1, "warmup": min(args.warmup, 3),
        "ms_per_step": 1000 * dt, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64/u32", "data": "synthetic",
        "config": {"workload": f"config {args.config}: {desc}", "products": count,
                   "num_primes": K},
        "cpu_baseline": {"value": v, "unit": "products/s", "cores": cores, "kind": "port",
                         "sample": f"first {n_done} of {count} products, oracle/bw_oracle.c "
                                   f"on {cores} threads, {dt:.1f} s"},
        "e2e": {"value": v, "unit": "products/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def serving_pool(count, seed, rank):
    """Distinct requests of the serving mix (operand pairs; squarings share
    one array)."""
    from birdwing_b200 import workloads
    rng = np.random.default_rng(seed + 1000 + 100 * rank)
    pool = []
    for la, lb, sq in workloads.serving_sizes(count, seed=seed + 100 * rank):
        a = workloads.rand_operand(rng, la)
        pool.append((a, a if sq else workloads.rand_operand(rng, lb)))
    return pool


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def run_open_loop(srv, pool, expect, rate, duration, seed, buffers=None):
    """Poisson arrivals at `rate` requests/s for `duration` seconds, cycling
    through the pool.  Latency = done - submit (library clock); every 32nd
    result is compared with GMP's as it is harvested (every pool entry is
    compared in the warm-up)."""
    rng = np.random.default_rng(seed)
    n_arr = int(rate * duration * 1.2) + 16
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_arr))
    arrivals = arrivals[arrivals < duration]
    # pool index -> free output buffers (pinned ones from `buffers` first)
    spare = {i: list(v) for i, v in (buffers or {}).items()}
    owner = {}                                  # ticket -> (pool index, buffer, check)
    lat, late, groups, bad, checked, done_in_window = [], [], [], 0, 0, 0
    unpinned = 0                                # outputs without a free pinned buffer
    t0 = time.perf_counter()

    def take_finished():
        nonlocal bad, checked, done_in_window
        while True:
            rec, outs = srv.harvest_arrays(8192)
            in_window = time.perf_counter() - t0 <= duration
            lat_ms = ((rec["done_us"] - rec["submit_us"]) * 1e-3).tolist()
            for t, st, g, l_ms in zip(rec["ticket"].tolist(), rec["status"].tolist(),
                                      rec["group_size"].tolist(), lat_ms):
                own = owner.pop(t, None)
                if own is None:
                    continue
                lat.append(l_ms)
                i, buf, chk = own
                if st != 0:
                    bad += 1
                elif chk:
                    checked += 1
                    if not np.array_equal(buf, expect[i]):
                        bad += 1
                groups.append(g)
                done_in_window += in_window
                spare.setdefault(i, []).append(buf)
            if len(rec) < 8192:
                break

    for k, t_arr in enumerate(arrivals):
        while True:
            now = time.perf_counter() - t0
            if now >= t_arr:
                break
            if t_arr - now > 2e-4:
                take_finished()
        i = k % len(pool)
        a, b = pool[i]
        free = spare.get(i)
        if free:
            out = free.pop()
        else:
            out = np.empty(len(a) + len(b), dtype=np.uint32)
            unpinned += 1
        late.append((time.perf_counter() - t0 - t_arr) * 1e3)
        owner[srv.submit(a, b, out=out)] = (i, out, k % 32 == 0)
    srv.drain()
    take_finished()
    wall = time.perf_counter() - t0
    return {"rate": rate, "submitted": len(arrivals), "completed": len(lat), "bad": bad,
            "checked_vs_gmp": checked, "submit_late_p99_ms": percentile(late, 99),
            "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99),
            "mean_ms": float(np.mean(lat)) if lat else None,
            "mean_group_size": float(np.mean(groups)) if groups else None,
            "products_per_s": len(lat) / wall, "drain_s": wall - duration,
            "completed_in_window": done_in_window, "unpinned_outputs": unpinned}


def run_plain_open_loop(pool, rate, duration, seed, max_wall):
    """The plain per-request path on the same arrival process: one thread
    serves requests in arrival order with bw_multiply_host_once (plan,
    context, multiply, teardown -- the drop-in host_multiply_merge).  Requests
    not served by max_wall count with their waiting time so far."""
    import ctypes

    from birdwing_b200 import _lib as L
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * duration * 1.2) + 16))
    arrivals = arrivals[arrivals < duration]
    lat, unserved = [], 0
    ms = ctypes.c_float()
    t0 = time.perf_counter()
    for k, t_arr in enumerate(arrivals):
        now = time.perf_counter() - t0
        if now < t_arr:
            time.sleep(t_arr - now)
            now = time.perf_counter() - t0
        if now > max_wall:
            unserved = len(arrivals) - k
            lat.extend((now - arrivals[k:]) * 1e3)
            break
        a, b = pool[k % len(pool)]
        out = np.empty(len(a) + len(b), dtype=np.uint32)
        L.check(L.lib.bw_multiply_host_once(
            ctypes.c_void_p(a.ctypes.data), a.size, ctypes.c_void_p(b.ctypes.data), b.size,
            ctypes.c_void_p(out.ctypes.data), out.size, L.BW_PATH_AUTO, ctypes.byref(ms)))
        lat.append((time.perf_counter() - t0 - t_arr) * 1e3)
    wall = time.perf_counter() - t0
    served = len(arrivals) - unserved
    return {"rate": rate, "submitted": len(arrivals), "served": served,
            "unserved_at_cutoff": unserved, "p50_ms": percentile(lat, 50),
            "p99_ms": percentile(lat, 99), "products_per_s": served / wall,
            "how": "bw_multiply_host_once per request (plan + context + multiply + teardown), "
                   "one server thread, arrival order"}


def bench_serving(args):
    import torch
    import torch.distributed as dist

    import birdwing_b200 as bw
    from oracle import gmp_ref

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    pool_n, seed, K, desc = SERVE_CONFIGS[args.config]
    pool = serving_pool(pool_n, seed, rank)
    expect = [gmp_ref.mul(a, b) for a, b in pool]

    # a serving client keeps its buffers in pinned memory: the server then
    # moves large operands and results by DMA without staging copies
    def pinned(x):
        return torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)

    pool = [(pinned(a), None if a is b else pinned(b)) for a, b in pool]
    pool = [(a, a if b is None else b) for a, b in pool]
    # four pinned output buffers per pool entry: a request whose entry has
    # none free gets a pageable one, which the server must stage (counted as
    # unpinned_outputs); with two, a brief latency spike at moderate rates ran
    # them out and the slower pageable results kept the queue growing
    buffers = {i: [pinned(np.zeros(len(a) + len(b), dtype=np.uint32)) for _ in range(4)]
               for i, (a, b) in enumerate(pool)}
    srv = bw.Server(num_primes=K)
    srv.prewarm(21)
    # warm-up: the whole pool, closed loop; the first pass checks every
    # result against GMP
    pool_ok = True
    for w in range(max(1, min(args.warmup, 3))):
        ts = {srv.submit(a, b, out=buffers[i][0]): i for i, (a, b) in enumerate(pool)}
        srv.drain()
        for d in srv.harvest(len(ts) + 16):
            if w == 0:
                pool_ok &= d["status"] == 0 and bool(
                    np.array_equal(d["out"], expect[ts[d["ticket"]]]))
    # capacity: the pool submitted at once, twice
    t0 = time.perf_counter()
    for _ in range(2):
        for i, (a, b) in enumerate(pool):
            srv.submit(a, b, out=buffers[i][0])
        srv.drain()
        srv.harvest(len(pool) + 16)
    cap = 2 * len(pool) / (time.perf_counter() - t0)
    fracs = [float(x) for x in args.rate_fracs.split(",")]
    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    sampler.start()
    st0 = srv.stats()
    sweep = [run_open_loop(srv, pool, expect, f * cap, args.duration, seed + 7 + j, buffers)
             for j, f in enumerate(fracs)]
    clocks = sampler.stop()
    st = srv.stats()
    srv.close()
    plain = None
    if not args.no_plain:
        plain = run_plain_open_loop(pool, fracs[0] * cap, min(args.duration, 10.0), seed + 99,
                                    max_wall=2 * min(args.duration, 10.0))
    # headline: the highest swept rate the server sustained (everything
    # submitted finished within 10% of the window after it closed)
    ok = [r for r in sweep if r["bad"] == 0 and r["drain_s"] <= 0.1 * args.duration]
    head = max(ok, key=lambda r: r["rate"]) if ok else sweep[0]
    vals = reduce_over_ranks([head["products_per_s"], head["p99_ms"] or 0.0], ["sum", "max"])
    if rank == 0:
        mean_in = float(np.mean([4 * (len(a) + (0 if a is b else len(b))) for a, b in pool]))
        mean_out = float(np.mean([4 * (len(a) + len(b)) for a, b in pool]))
        line = {
            "metric": "products/s", "value": vals[0], "unit": "products/s",
            "n_gpus": world, "steps": head["completed"], "warmup": args.warmup,
            "ms_per_step": 1000.0 / vals[0], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"config {args.config}: {desc}", "pool": pool_n,
                       "num_primes": K, "duration_s": args.duration,
                       "rates": [r["rate"] for r in sweep], "capacity_closed_loop": cap,
                       "l2": "operands streamed from host per request",
                       "parallelism": f"replicas x{world}"},
            "latency_ms": {"p50": head["p50_ms"], "p99": vals[1], "at_rate": head["rate"]},
            "sweep": sweep,
            "server_stats": st,
            "plain_per_request": plain,
            "correct_vs_gmp": pool_ok and all(r["bad"] == 0 for r in sweep),
            "e2e": {"value": vals[0], "unit": "products/s",
                    "h2d_bytes_per_step": mean_in, "d2h_bytes_per_step": mean_out,
                    "note": "every request is host buffers in, host buffers out"},
            "gpu_launches": st["kernel_launches"] - st0["kernel_launches"],
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:   # the CPU baseline runs at N = 1 only
            line["cpu_baseline"] = cpu_baseline_items([(64, a, b) for a, b in pool], K)
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_reference_serving(args):
    """--impl reference on the serving configuration: the oracle serves the
    request pool in order on all host threads (a bounded sample)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    pool_n, seed, K, desc = SERVE_CONFIGS[args.config]
    pool = serving_pool(pool_n, seed, 0)
    cores = os.cpu_count() or 1
    oracle.lib.oracle_set_threads(cores)
    lat, t0 = [], time.perf_counter()
    for a, b in pool:
        t1 = time.perf_counter()
        oracle.multiply(a, b, 64, K)
        lat.append((time.perf_counter() - t1) * 1e3)
        if time.perf_counter() - t0 >= 120.0:
            break
    dt = time.perf_counter() - t0
    v = len(lat) / dt
    line = {
        "impl": "reference", "metric": "products/s", "value": v, "unit": "products/s",
        "n_gpus": args.gpus, "steps": len(lat), "warmup": 0, "ms_per_step": 1000.0 / v,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic", "config": {"workload": f"config {args.config}: {desc}",
                                        "pool": pool_n, "num_primes": K},
        "latency_ms": {"p50": percentile(lat, 50), "p99": percentile(lat, 99),
                       "note": "service time per request, closed loop (no queueing)"},
        "cpu_baseline": {"value": v, "unit": "products/s", "cores": cores, "kind": "port",
                         "sample": f"first {len(lat)} of {pool_n} pool requests, "
                                   f"oracle/bw_oracle.c on {cores} threads, {dt:.1f} s"},
        "e2e": {"value": v, "unit": "products/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def bench_intpeak(args):
    """Integer-pipe ceiling of both prime paths (bw_butterfly_rate): the
    transforms' own forward and inverse butterflies from registers, no memory
    traffic, swept over 2/4/8 CTAs of 256 threads per SM, best of 3 each.
    Reported per second and per SM-cycle at the SM clock sampled during the
    timed launches; the plain configurations' int_floor divides their
    butterflies by the same rate."""
    import torch

    from birdwing_b200 import _lib as L
    if args.impl == "reference":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has no integer-throughput probe: its transforms "
                          "are the absent GPU-NTT library's"}))
        return
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.05)
    paths, t0 = {}, time.perf_counter()
    for name, path in (("p32", L.BW_PATH_P32), ("p64", L.BW_PATH_P64)):
        best, sweep = butterfly_rate(path)
        paths[name] = {"butterflies_per_s": best,
                       "ctas_per_sm": max(sweep, key=sweep.get),
                       "sweep": {str(c): r for c, r in sweep.items()}}
    t1 = time.perf_counter()
    clocks.region(t0, t1)
    ck = clocks.stop()
    mhz = ck.get("sm_mhz") or 0.0
    for v in paths.values():
        v["per_sm_cycle"] = v["butterflies_per_s"] / (sms * mhz * 1e6) if mhz else None
    line = {
        "metric": "butterflies/s", "value": paths["p64"]["butterflies_per_s"],
        "unit": "butterflies/s", "n_gpus": 1, "steps": 3, "warmup": 1,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic",
        "config": {"workload": "intpeak: 16 residues per thread, two radix-16 forward rounds "
                               "and one inverse round per iteration (96 butterflies), 2000 "
                               "iterations, 256-thread CTAs",
                   "sms": sms},
        "paths": paths, "p32_over_p64": paths["p32"]["butterflies_per_s"]
        / paths["p64"]["butterflies_per_s"],
        "gpu_launches": 2 * 3 * 3 * 2, "clocks": ck,
    }
    print(json.dumps(line))


def main():
    args = parse()
    if args.config == "intpeak":
        bench_intpeak(args)
        return
    if args.config in SERVE_CONFIGS:
        if args.impl == "reference":
            run_reference_serving(args)
        else:
            bench_serving(args)
        return
    if args.config in BATCH_CONFIGS:
        if args.impl == "reference":
            run_reference_batch(args)
        else:
            bench_batch(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    bench_plain(args)


def fixed_model(cfg):
    """The fixed algorithmic byte model of a plain configuration (SURVEY-style
    12*K*n*w + in + out, 9*K*n*w + in + out when squaring) evaluated on the
    workload as the reference states it (its coefficient width, prime count
    and prime width), whatever algorithm the library chose.  Returns (bytes,
    K, n, w)."""
    la, lb, path, K, square, _ = CONFIGS[cfg]
    cpw = 2 if path == 32 else 1
    log_n = max(4, ((la + (la if square else lb)) * cpw - 2).bit_length())
    n, w = 1 << log_n, (8 if path == 64 else 4)
    io = 4 * (la + (0 if square else lb)) + 4 * (la + lb)
    return (9 if square else 12) * K * n * w + io, K, n, w


def plain_launches_of(info, la, lb):
    """Kernels one plain product launches: the forward column, row and inverse
    column passes (two middle-column passes more in the three-pass
    schedule), and Garner + carry: the boundary pre-pass, the words pass and
    the carry fix when the output spans more than one 2048-word tile, else
    the words pass alone."""
    log_r2 = info["log_n"] - info["log_rows"] - info["log_cols"]
    return 3 + (2 if log_r2 > 0 else 0) + (3 if la + lb > 2048 else 1)


def plan_butterflies(info, square):
    """Butterflies of one product: T transforms (3, or 2 when squaring) of K
    primes, each (n/2) log2 n."""
    t = 2 if square else 3
    return t * info["num_primes"] * (1 << (info["log_n"] - 1)) * info["log_n"]


def butterfly_rate(path, iters=2000):
    """Integer-pipe ceiling of the path's butterflies (bw_butterfly_rate):
    butterflies per second with nothing else running, best of 3 at each of
    2/4/8 CTAs per SM.  Returns (best rate, {ctas_per_sm: rate})."""
    import ctypes

    from birdwing_b200 import _lib as L
    sweep = {}
    for cps in (2, 4, 8):
        best = None
        for _ in range(3):
            ms, bf = ctypes.c_float(), ctypes.c_double()
            L.check(L.lib.bw_butterfly_rate(path, iters, cps, ctypes.byref(ms), ctypes.byref(bf)))
            r = bf.value / (ms.value * 1e-3)
            best = r if best is None else max(best, r)
        sweep[cps] = best
    return max(sweep.values()), sweep


def run_sub_bench(extra, timeout):
    """Run this script once more as a child process (one GPU, no torchrun
    variables) and return its JSON line, or {"error": ...}."""
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "LOCAL_RANK", "WORLD_SIZE", "LOCAL_WORLD_SIZE", "MASTER_ADDR",
                        "MASTER_PORT", "GROUP_RANK", "ROLE_RANK", "TORCHELASTIC_RUN_ID")}
    cmd = [sys.executable, os.path.abspath(__file__)] + extra
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout} s", "cmd": " ".join(extra)}
    for ln in reversed(r.stdout.strip().splitlines()):
        if ln.startswith("{"):
            try:
                return json.loads(ln)
            except ValueError:
                break
    return {"error": f"exit {r.returncode}: {r.stderr.strip()[-400:]}", "cmd": " ".join(extra)}


def batched_summary(line):
    if "error" in line:
        return line
    pl = line.get("plain_loop") or {}
    return {"workload": line["config"]["workload"], "value": line["value"],
            "unit": line["unit"], "ms_per_step": line["ms_per_step"],
            "plain_loop_value": pl.get("value"),
            "batched_over_plain": line.get("batched_over_plain"),
            "e2e_value": line["e2e"]["value"], "correct_vs_gmp": line["correct_vs_gmp"],
            "buckets": line["config"]["buckets"], "clocks": line.get("clocks"),
            "cmd": "python bench.py --config 3 --steps 10 --warmup 3 --e2e-steps 2 "
                   "--no-cpu-baseline"}


def serving_summary(line):
    if "error" in line:
        return line
    plain = line.get("plain_per_request") or {}
    return {"workload": line["config"]["workload"], "value": line["value"],
            "unit": line["unit"], "p50_ms": line["latency_ms"]["p50"],
            "p99_ms": line["latency_ms"]["p99"], "at_rate": line["latency_ms"]["at_rate"],
            "capacity_closed_loop": line["config"]["capacity_closed_loop"],
            "plain_per_request": {k: plain.get(k) for k in ("rate", "products_per_s", "p50_ms",
                                                            "p99_ms", "unserved_at_cutoff")},
            "correct_vs_gmp": line["correct_vs_gmp"], "clocks": line.get("clocks"),
            "cmd": "python bench.py --config 5 --duration 4 --rate-fracs 0.45 --warmup 1 "
                   "--no-cpu-baseline"}


def bench_plain(args):
    import torch
    import torch.distributed as dist

    import birdwing_b200 as bw

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    cfg = args.config
    la, lb, _, _, square, desc = CONFIGS[cfg]
    _, _, ppath, pk, pflags = plain_plan_args(cfg)
    a, b = operands(cfg, rank)
    plan = bw.Plan(la, lb, ppath, pk, log_cols=args.log_cols, flags=pflags | args.plan_flags)
    info = plan.info
    K, n, path = info["num_primes"], plan.N, info["path"]
    w = 8 if path == 64 else 4
    ctx = bw.Context(plan)
    stream = torch.cuda.ExternalStream(ctx.stream)

    # inputs resident in HBM for the device-time measurement
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = da if square else torch.from_numpy(b.view(np.int32)).cuda()
    dc = torch.empty(la + lb, dtype=torch.int32, device="cuda")
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")

    def make_step(c):
        def step(timing):
            return c.multiply_device(da.data_ptr(), la, db.data_ptr(), lb, dc.data_ptr(),
                                     la + lb, timing=timing)
        return step

    def check_product():
        got = dc.cpu().numpy().view(np.uint32)
        if cfg in CPU_SAMPLE_WORDS:
            return residue_check(a, b, got), "residues mod 2^64 and three random 61-bit primes"
        from oracle import gmp_ref
        return bool((got == gmp_ref.mul(a, b)).all()), "GMP mpz_mul"

    def timed_products(c, st, steps, sampler=None):
        """steps whole products back to back on the context stream (graph
        replays), L2 flushed before each; returns the per-step event times."""
        step = make_step(c)
        ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(steps):
            with torch.cuda.stream(st):
                flush.fill_(i)                       # evict L2 between steps
                ev0[i].record(st)
            step(False)
            with torch.cuda.stream(st):
                ev1[i].record(st)
        torch.cuda.synchronize()
        if sampler:
            sampler.region(t0, time.perf_counter())
        return [e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1)]

    def stage_means(c, st, reps):
        """Per-stage device times (events between the kernels, direct
        launches), outside the timed region."""
        step = make_step(c)
        stage = {k: [] for k in ("fwd_ms", "mul_ms", "intt_ms", "crt_carry_ms")}
        for i in range(reps):
            with torch.cuda.stream(st):
                flush.fill_(i)
            t = step(True)
            for k in stage:
                stage[k].append(t[k])
        return {k: statistics.mean(v) for k, v in stage.items()}

    step = make_step(ctx)
    for _ in range(max(3, args.warmup)):
        step(False)
    ctx.sync()
    # correctness of the benchmarked product (once, outside the timed region)
    ok, check = check_product() if rank == 0 else (True, "")
    device_bytes = (info["plan_device_bytes"] + info["ctx_device_bytes"] +
                    4 * (la + (0 if square else lb)) + 4 * (la + lb))

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.05)
    per_step = timed_products(ctx, stream, args.steps, sampler)
    stage = stage_means(ctx, stream, max(3, min(args.steps, 10)))
    clocks = sampler.stop()
    barrier()
    ctx.sync()
    total_ms = reduce_over_ranks([sum(per_step)], ["max"])[0]

    # end to end through the C ABI with pinned host buffers
    ha = torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32)
    hb = ha if square else torch.from_numpy(b.view(np.int32)).pin_memory().numpy().view(np.uint32)
    hc = torch.empty(la + lb, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    for _ in range(2):
        ctx.multiply(ha, hb, out=hc)
    barrier()
    # blocking: one call per product (copy in, compute, copy out, wait)
    e2e_ms = []
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        ctx.multiply(ha, hb, out=hc)
        e2e_ms.append(1000 * (time.perf_counter() - t0))
    e2e_block_total = reduce_over_ranks([sum(e2e_ms)], ["max"])[0]
    # blocking from pageable numpy arrays: the drop-in host_multiply_merge case
    pc = np.empty(la + lb, dtype=np.uint32)
    ctx.multiply(a, b, out=pc)
    e2e_pg = []
    for _ in range(min(args.e2e_steps, 3)):
        t0 = time.perf_counter()
        ctx.multiply(a, b, out=pc)
        e2e_pg.append(1000 * (time.perf_counter() - t0))
    e2e_pg_total = reduce_over_ranks([sum(e2e_pg)], ["max"])[0]
    # pipelined: contexts of one plan used in turn (BW_PTR_HOST_ASYNC); the
    # library orders each stage after the previous product's same stage, so one
    # product copies in while another computes and a third copies out (two
    # contexts for products whose contexts take tens of GiB).  Every product
    # still copies its operands in and its result out; the count covers the
    # pipeline's fill and drain.
    ring = [(ctx, hc)]
    for _ in range(3 if n < (1 << 27) else 1):
        ring.append((bw.Context(plan),
                     torch.empty(la + lb, dtype=torch.int32).pin_memory().numpy().view(np.uint32)))
    for c_, o_ in ring:
        c_.multiply_async(ha, hb, o_)
    for c_, _ in ring:
        c_.sync()
    e2e_steps = max(args.e2e_steps, 24 if n < (1 << 27) else 6)
    barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        c_, o_ = ring[i % len(ring)]
        if i >= len(ring):
            c_.sync()                      # the previous product on this context is done
        c_.multiply_async(ha, hb, o_)
    for c_, _ in ring:
        c_.sync()
    e2e_pipe_total = reduce_over_ranks([1000 * (time.perf_counter() - t0)], ["max"])[0]
    ok_e2e = True
    if rank == 0:
        if cfg in CPU_SAMPLE_WORDS:
            ok_e2e = all(residue_check(a, b, o_) for _, o_ in ring)
        else:
            from oracle import gmp_ref
            want = gmp_ref.mul(a, b)
            ok_e2e = all(bool((o_ == want).all()) for _, o_ in ring)
    for c_, _ in ring[1:]:
        c_.close()

    # the workload as the reference states it (its coefficient width and
    # prime count), when the library's own plan differs: same operands, same
    # timing, rank 0 of a single-GPU run
    def side_record(which, e2e=False):
        """The same product under another plan of the table (same operands,
        same timing): the workload as the reference states it, or the other
        prime path (e2e: also end to end from pinned host buffers, four
        contexts in turn, as the headline's `e2e`)."""
        sp = plain_plan_args(cfg, which)
        with bw.Plan(*sp[:4], flags=sp[4]) as splan, bw.Context(splan) as sctx:
            sst = torch.cuda.ExternalStream(sctx.stream)
            sstep = make_step(sctx)
            for _ in range(3):
                sstep(False)
            sctx.sync()
            sok, _ = check_product()
            sper = timed_products(sctx, sst, max(args.steps, 20))
            sstage = stage_means(sctx, sst, 5)
            sctx.sync()
            si = splan.info
            rec = {"algorithm": algorithm_of(si), "path": si["path"],
                   "coeff_bits": si["coeff_bits"], "num_primes": si["num_primes"],
                   "log_n": si["log_n"], "ms_per_step": sum(sper) / len(sper),
                   "value": len(sper) / (sum(sper) * 1e-3), "unit": "products/s",
                   "stage_ms": sstage, "correct_vs_gmp": sok, "_info": si}
            if e2e:
                ring = [(sctx, hc)] + [
                    (bw.Context(splan),
                     torch.empty(la + lb, dtype=torch.int32).pin_memory().numpy().view(np.uint32))
                    for _ in range(3)]
                for c_, o_ in ring:
                    c_.multiply_async(ha, hb, o_)
                for c_, _ in ring:
                    c_.sync()
                steps = max(args.e2e_steps, 24)
                t0 = time.perf_counter()
                for i in range(steps):
                    c_, o_ = ring[i % len(ring)]
                    if i >= len(ring):
                        c_.sync()
                    c_.multiply_async(ha, hb, o_)
                for c_, _ in ring:
                    c_.sync()
                dt = time.perf_counter() - t0
                from oracle import gmp_ref
                want = gmp_ref.mul(a, b)
                rec["e2e"] = {"value": steps / dt, "unit": "products/s",
                              "h2d_bytes_per_step": 4 * (la + (0 if square else lb)),
                              "d2h_bytes_per_step": 4 * (la + lb),
                              "correct_vs_gmp": all(bool((o_ == want).all()) for _, o_ in ring),
                              "how": "bw_multiply(BW_PTR_HOST_ASYNC) on four contexts of one "
                                     "plan in turn from pinned host buffers, wall clock"}
                for c_, _ in ring[1:]:
                    c_.close()
            return rec

    literal = None
    if world == 1 and PLAIN[cfg]["literal"] != PLAIN[cfg]["plan"]:
        literal = side_record("literal")
        literal.pop("_info")
    # the other prime path for the same product (the 32-bit path with 64-bit
    # coefficients for the 2^28-bit workloads)
    other = None
    if world == 1 and PLAIN[cfg].get("other"):
        other = side_record("other", e2e=cfg not in CPU_SAMPLE_WORDS)

    if rank == 0:
        ms = total_ms / args.steps
        mb = model_bytes(la, lb, n, K, w, square)
        dom = max(stage, key=stage.get)
        kernel_names = {"fwd_ms": "k_fwd_col", "mul_ms": "k_row", "intt_ms": "k_inv_col",
                        "crt_carry_ms": "k_garner_carry"}
        peak, peak_kind = load_peaks()
        achieved = mb[dom] / (stage[dom] * 1e-3) / 1e9
        own_model = sum(mb.values())
        fixed, fk, fn, fw = fixed_model(cfg)
        line = {
            "metric": "products/s", "value": job_throughput(args.steps, world, total_ms),
            "unit": "products/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64" if path == 64 else "u32", "data": "synthetic",
            "config": {"workload": f"config {cfg}: {desc}", "algorithm": algorithm_of(info),
                       "words_a": la, "words_b": lb, "path": path, "num_primes": K,
                       "coeff_bits": info["coeff_bits"], "log_n": plan.logN,
                       "log_cols": info["log_cols"], "plan_flags": pflags | args.plan_flags,
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas x{world}"},
            "correct_vs_gmp": ok,
            "correctness_check": check,
            "hbm_footprint_bytes": device_bytes,
            "stage_ms": stage,
            "roofline": {"bound": "hbm", "kernel": kernel_names[dom], "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "traffic": load_traffic(cfg, kernel_names[dom]),
                         "algorithmic_bytes": mb[dom],
                         "bytes_model": "the chosen algorithm's K*n*w per kernel"},
            "product_roofline": {
                "fixed_model_bytes": fixed,
                "fixed_model": f"12*K*n*w + in + out at the workload's stated K={fk}, "
                               f"n=2^{fn.bit_length() - 1}, w={fw}",
                "achieved": fixed / (ms * 1e-3) / 1e9, "unit": "GB/s",
                "frac": fixed / (ms * 1e-3) / 1e9 / peak,
                "own_model_bytes": own_model,
                "own_model_frac": own_model / (ms * 1e-3) / 1e9 / peak},
            "e2e": {"value": job_throughput(e2e_steps, world, e2e_pipe_total),
                    "unit": "products/s", "h2d_bytes_per_step": 4 * (la + (0 if square else lb)),
                    "d2h_bytes_per_step": 4 * (la + lb) + 4,
                    "how": "bw_multiply(BW_PTR_HOST_ASYNC) on four contexts of one plan in "
                           "turn (stage-ordered copy-in / kernels / copy-out) from pinned host "
                           "buffers; wall clock over all steps with the pipeline's fill and "
                           "drain",
                    "blocking_value": job_throughput(args.e2e_steps, world, e2e_block_total),
                    "blocking_pageable_value": job_throughput(min(args.e2e_steps, 3), world,
                                                              e2e_pg_total),
                    "correct_vs_gmp": ok_e2e},
            "gpu_launches": plain_launches_of(info, la, lb) * args.steps,
            "clocks": clocks,
        }
        if literal:
            literal["product_roofline_frac"] = fixed / (literal["ms_per_step"] * 1e-3) / 1e9 / peak
            line["literal_config"] = literal
        if other:
            oi = other.pop("_info")
            other["product_roofline_frac"] = fixed / (other["ms_per_step"] * 1e-3) / 1e9 / peak
            orate, _ = butterfly_rate(oi["path"])
            ofloor = plan_butterflies(oi, square) / orate * 1e3
            other["int_floor"] = {"butterflies": plan_butterflies(oi, square),
                                  "butterflies_per_s": orate, "floor_ms": ofloor}
            other["int_floor_frac"] = ofloor / other["ms_per_step"]
            line["other_path"] = other
        if world == 1:
            # integer-pipe floor: the plan's butterflies at the rate the
            # path's butterflies reach with nothing else running
            rate, _ = butterfly_rate(path)
            bfly = plan_butterflies(info, square)
            floor_ms = bfly / rate * 1e3
            line["int_floor"] = {"butterflies": bfly, "butterflies_per_s": rate,
                                 "floor_ms": floor_ms, "frac": floor_ms / ms,
                                 "how": "bw_butterfly_rate: the path's own forward and inverse "
                                        "butterflies from registers, best over 2/4/8 CTAs per SM "
                                        "(bench.py --config intpeak)"}
            line["int_floor_frac"] = floor_ms / ms
        if not args.no_cpu_baseline and world == 1:   # the CPU baseline runs at N = 1 only
            line["cpu_baseline"] = cpu_baseline(cfg)
        if cfg == "2" and world == 1 and not args.no_sub:
            # the metric's other halves, each in a child process of its own
            line["batched"] = batched_summary(run_sub_bench(
                ["--config", "3", "--steps", "10", "--warmup", "3", "--e2e-steps", "2",
                 "--no-cpu-baseline"], timeout=300))
            line["serving"] = serving_summary(run_sub_bench(
                ["--config", "5", "--duration", "4", "--rate-fracs", "0.45", "--warmup", "1",
                 "--no-cpu-baseline"], timeout=300))
        print(json.dumps(line))
    ctx.close()
    plan.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
