"""Size sweep with the reference benchmark's CSV schema.

Writes the columns of the reference's full-multiply benchmark
(bench/gpu_full_multiply_benchmark.cpp:397-404), so its plotting script
(scripts/plot_bench.py) reads these runs unchanged:

    python -m birdwing_b200.sweep --pipeline hybrid --L 1024,65536,1048576 --csv out.csv

Pipelines (the reference's names): "32" = 32-bit prime path, u32 limbs;
"hybrid" = 64-bit prime path, u32 limbs; "64bit" = 64-bit prime path, u64
limbs (passed to the library as twice as many u32 words).  L counts host
limbs of each operand; an argument below 64 means 2^L_arg limbs, as the
reference resolves it (bench/gpu_full_multiply_benchmark.cpp:111-116).

How the stage columns map onto this pipeline (its kernels fuse stages the
reference runs separately):
  h2d_mean_ms           copy-in of both operands
  fwd_pad_ntt_mean_ms   limb split + virtual zero pad + forward column pass
                        of both operands (one launch); the _a/_b columns get
                        half of it each
  ingress_fwd_mean_ms   h2d + fwd_pad_ntt
  mul_mean_ms           the fused row pass: forward rows, pointwise product,
                        inverse rows
  intt_mean_ms          the inverse column pass
  crt_mean_ms           fused Garner + carry (one kernel); carry_mean_ms is 0
  d2h_mean_ms           copy-out of the product
  setup_precompute_ms   bw_plan_create (host tables and their upload), with
                        setup_upload_ms 0; setup_alloc_ms bw_ctx_create
Columns with no counterpart (the precompute and upload sub-steps) are 0.
"""
import argparse
import csv
import os
import statistics
import time

import numpy as np

HEADER = [
    "pipeline", "host_limb_bits", "operand_bits", "L_arg", "L", "N", "logN", "warmup", "iters",
    "mean_ms", "stddev_ms", "min_ms", "max_ms",
    "setup_pinned_ms", "setup_precompute_ms", "setup_upload_ms", "setup_alloc_ms",
    "pre_factors_ms", "pre_params_ms", "pre_twiddle_host_ms", "pre_garner_host_ms",
    "upload_twiddle_ms", "upload_mod_constants_ms", "upload_garner_ms",
    "teardown_free_ctx_ms", "teardown_free_pre_ms", "teardown_free_pinned_ms",
    "ingress_fwd_mean_ms", "h2d_mean_ms", "fwd_pad_ntt_mean_ms", "fwd_pad_ntt_a_mean_ms",
    "fwd_pad_ntt_b_mean_ms",
    "mul_mean_ms", "intt_mean_ms", "crt_mean_ms", "carry_mean_ms", "d2h_mean_ms",
]

PIPELINES = {"32": (32, 32), "hybrid": (64, 32), "64bit": (64, 64)}  # (prime path, limb bits)


def resolve_limbs(L_arg):
    """Limb count of an L argument: below 64 it is a power of two."""
    return 1 << L_arg if L_arg < 64 else L_arg


def make_row(pipeline, L_arg, log_n, warmup, totals, stages, setup, teardown):
    """One CSV row (dict) from measured times in ms.  stages: list of
    bw_timing dicts; setup: pinned/precompute/alloc; teardown: ctx/pre/pinned."""
    limb_bits = PIPELINES[pipeline][1]
    L = resolve_limbs(L_arg)

    def mean(k):
        return statistics.mean(t[k] for t in stages) if stages else 0.0

    fwd = mean("fwd_ms")
    row = dict.fromkeys(HEADER, 0.0)
    row.update({
        "pipeline": pipeline, "host_limb_bits": limb_bits, "operand_bits": L * limb_bits,
        "L_arg": L_arg, "L": L, "N": 1 << log_n, "logN": log_n, "warmup": warmup,
        "iters": len(totals),
        "mean_ms": statistics.mean(totals),
        "stddev_ms": statistics.pstdev(totals),
        "min_ms": min(totals), "max_ms": max(totals),
        "setup_pinned_ms": setup.get("pinned", 0.0),
        "setup_precompute_ms": setup.get("precompute", 0.0),
        "setup_alloc_ms": setup.get("alloc", 0.0),
        "teardown_free_ctx_ms": teardown.get("ctx", 0.0),
        "teardown_free_pre_ms": teardown.get("pre", 0.0),
        "teardown_free_pinned_ms": teardown.get("pinned", 0.0),
        "h2d_mean_ms": mean("h2d_ms"),
        "fwd_pad_ntt_mean_ms": fwd, "fwd_pad_ntt_a_mean_ms": fwd / 2,
        "fwd_pad_ntt_b_mean_ms": fwd / 2,
        "ingress_fwd_mean_ms": mean("h2d_ms") + fwd,
        "mul_mean_ms": mean("mul_ms"), "intt_mean_ms": mean("intt_ms"),
        "crt_mean_ms": mean("crt_carry_ms"), "carry_mean_ms": 0.0,
        "d2h_mean_ms": mean("d2h_ms"),
    })
    return row


def product_ok(a, b, c, count=2, seed=61):
    """Whether c = a*b, from residues mod 2^64 and mod `count` random 61-bit
    probable primes (linear time, so it runs at every swept size)."""
    def as_int(w):
        return int.from_bytes(np.ascontiguousarray(w).view(np.uint8).tobytes(), "little")
    A, B, C = as_int(a), as_int(b), as_int(c)
    rng = np.random.default_rng(seed)
    mods = [1 << 64]
    while len(mods) < count + 1:
        m = int(rng.integers(1 << 60, 1 << 61)) | 1
        if pow(3, m - 1, m) == 1:
            mods.append(m)
    return all(C % m == (A % m) * (B % m) % m for m in mods)


def write_csv(path, rows, append=False):
    """Write rows with the reference's header (once, when the file is new or
    empty), numbers with six decimals as the reference writes them."""
    header = not append or not os.path.exists(path) or os.path.getsize(path) == 0
    with open(path, "a" if append else "w", newline="") as f:
        w = csv.writer(f)
        if header:
            w.writerow(HEADER)
        for r in rows:
            w.writerow([f"{r[k]:.6f}" if isinstance(r[k], float) else r[k] for k in HEADER])


def measure(pipeline, L_arg, warmup=2, iters=5, seed=1234):
    """Time one size through the C ABI: setup (pin, plan, context), iters
    blocking products from pinned host buffers with per-stage events, and
    teardown.  The last product is checked before the row is returned.
    None when the pipeline's primes do not reach this size."""
    import torch

    import birdwing_b200 as bw
    path, limb_bits = PIPELINES[pipeline]
    words = resolve_limbs(L_arg) * limb_bits // 32
    if not bw.size_supported(words, words, path)[0]:
        return None
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 1 << 32, words, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 1 << 32, words, dtype=np.uint64).astype(np.uint32)
    a[-1] |= np.uint32(1 << 31)
    b[-1] |= np.uint32(1 << 31)
    t0 = time.perf_counter()
    ha = torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32)
    hb = torch.from_numpy(b.view(np.int32)).pin_memory().numpy().view(np.uint32)
    hc = torch.empty(2 * words, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    t1 = time.perf_counter()
    plan = bw.Plan(words, words, path)
    t2 = time.perf_counter()
    ctx = bw.Context(plan)
    t3 = time.perf_counter()
    for _ in range(warmup):
        ctx.multiply(ha, hb, out=hc)
    totals, stages = [], []
    for _ in range(iters):
        s = time.perf_counter()
        _, t = ctx.multiply(ha, hb, out=hc, timing=True)
        totals.append(1000 * (time.perf_counter() - s))
        stages.append(t)
    t4 = time.perf_counter()
    if not product_ok(ha, hb, hc):
        raise RuntimeError(f"{pipeline} L_arg={L_arg}: product check failed")
    t4b = time.perf_counter()
    ctx.close()
    t5 = time.perf_counter()
    log_n = plan.logN
    plan.close()
    t6 = time.perf_counter()
    del ha, hb, hc
    t7 = time.perf_counter()
    return make_row(pipeline, L_arg, log_n, warmup, totals, stages,
                    {"pinned": 1000 * (t1 - t0), "precompute": 1000 * (t2 - t1),
                     "alloc": 1000 * (t3 - t2)},
                    {"ctx": 1000 * (t5 - t4b), "pre": 1000 * (t6 - t5),
                     "pinned": 1000 * (t7 - t6)})


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--pipeline", default="hybrid", choices=sorted(PIPELINES))
    ap.add_argument("--L", default=",".join(str(i) for i in range(6, 23)),
                    help="comma-separated host-limb counts per operand (below 64: log2)")
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--iters", type=int, default=5)
    ap.add_argument("--csv", default="gpu_full_multiply.csv")
    ap.add_argument("--append", action="store_true")
    args = ap.parse_args(argv)
    rows = []
    for x in args.L.split(","):
        r = measure(args.pipeline, int(x), args.warmup, args.iters)
        if r is None:
            print(f"{args.pipeline:>7} L_arg={x}: beyond this pipeline's transform length")
        else:
            rows.append(r)
    write_csv(args.csv, rows, args.append)
    for r in rows:
        print(f"{r['pipeline']:>7} L={r['L']:>9} N=2^{r['logN']:<2} mean {r['mean_ms']:.3f} ms")


if __name__ == "__main__":
    main()
