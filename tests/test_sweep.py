"""The size sweep writes the reference benchmark's CSV schema
(bench/gpu_full_multiply_benchmark.cpp:397-404) with the reference's
statistics (population stddev, :170-173) and L resolution (:111-116), and
holds the columns its plotting script requires (scripts/plot_bench.py:15-17,
53-60, 157-161)."""
import csv
import statistics

import numpy as np
import pytest

from birdwing_b200 import sweep

# The header line exactly as the reference writes it.
REFERENCE_HEADER = (
    "pipeline,host_limb_bits,operand_bits,L_arg,L,N,logN,warmup,iters,"
    "mean_ms,stddev_ms,min_ms,max_ms,"
    "setup_pinned_ms,setup_precompute_ms,setup_upload_ms,setup_alloc_ms,"
    "pre_factors_ms,pre_params_ms,pre_twiddle_host_ms,pre_garner_host_ms,"
    "upload_twiddle_ms,upload_mod_constants_ms,upload_garner_ms,"
    "teardown_free_ctx_ms,teardown_free_pre_ms,teardown_free_pinned_ms,"
    "ingress_fwd_mean_ms,h2d_mean_ms,fwd_pad_ntt_mean_ms,fwd_pad_ntt_a_mean_ms,"
    "fwd_pad_ntt_b_mean_ms,"
    "mul_mean_ms,intt_mean_ms,crt_mean_ms,carry_mean_ms,d2h_mean_ms"
)
PLOT_CORE = {"L_arg", "L", "N", "mean_ms", "stddev_ms", "min_ms", "max_ms"}
PLOT_STACK = ["ingress_fwd_mean_ms", "mul_mean_ms", "intt_mean_ms", "crt_mean_ms",
              "carry_mean_ms", "d2h_mean_ms"]


def stage(h2d, fwd, mul, intt, crt, d2h):
    return {"h2d_ms": h2d, "fwd_ms": fwd, "mul_ms": mul, "intt_ms": intt,
            "crt_carry_ms": crt, "d2h_ms": d2h, "total_ms": h2d + fwd + mul + intt + crt + d2h}


def test_header_is_the_reference_header():
    assert ",".join(sweep.HEADER) == REFERENCE_HEADER


def test_limb_resolution():
    assert sweep.resolve_limbs(6) == 64
    assert sweep.resolve_limbs(22) == 1 << 22
    assert sweep.resolve_limbs(64) == 64
    assert sweep.resolve_limbs(1000) == 1000


def test_row_values():
    totals = [1.0, 2.0, 4.0]
    stages = [stage(0.1, 0.2, 0.3, 0.4, 0.5, 0.6), stage(0.3, 0.4, 0.5, 0.6, 0.7, 0.8)]
    r = sweep.make_row("64bit", 10, 12, 3, totals, stages,
                       {"pinned": 1.5, "precompute": 2.5, "alloc": 3.5},
                       {"ctx": 0.1, "pre": 0.2, "pinned": 0.3})
    assert r["pipeline"] == "64bit" and r["host_limb_bits"] == 64
    assert r["L_arg"] == 10 and r["L"] == 1024 and r["operand_bits"] == 1024 * 64
    assert r["N"] == 4096 and r["logN"] == 12 and r["warmup"] == 3 and r["iters"] == 3
    assert r["mean_ms"] == pytest.approx(7 / 3)
    assert r["stddev_ms"] == pytest.approx(statistics.pstdev(totals))
    assert (r["min_ms"], r["max_ms"]) == (1.0, 4.0)
    assert r["h2d_mean_ms"] == pytest.approx(0.2)
    assert r["fwd_pad_ntt_mean_ms"] == pytest.approx(0.3)
    assert r["fwd_pad_ntt_a_mean_ms"] + r["fwd_pad_ntt_b_mean_ms"] == pytest.approx(0.3)
    assert r["ingress_fwd_mean_ms"] == pytest.approx(0.5)
    assert r["mul_mean_ms"] == pytest.approx(0.4) and r["intt_mean_ms"] == pytest.approx(0.5)
    assert r["crt_mean_ms"] == pytest.approx(0.6) and r["carry_mean_ms"] == 0.0
    assert r["d2h_mean_ms"] == pytest.approx(0.7)
    assert r["setup_precompute_ms"] == 2.5 and r["setup_upload_ms"] == 0.0
    assert r["teardown_free_pinned_ms"] == 0.3


def test_csv_round_trip_and_append(tmp_path):
    path = tmp_path / "s.csv"
    r32 = sweep.make_row("32", 6, 7, 1, [0.5], [stage(*[0.01] * 6)], {}, {})
    rh = sweep.make_row("hybrid", 4096, 13, 1, [0.5, 0.7], [stage(*[0.02] * 6)], {}, {})
    sweep.write_csv(str(path), [r32])
    sweep.write_csv(str(path), [rh], append=True)
    text = path.read_text().splitlines()
    assert text[0] == REFERENCE_HEADER
    assert sum(1 for line in text if line.startswith("pipeline,")) == 1
    with open(path, newline="") as f:
        rd = csv.DictReader(f)
        assert PLOT_CORE.issubset(rd.fieldnames) and "pipeline" in rd.fieldnames
        assert set(PLOT_STACK).issubset(rd.fieldnames)
        rows = list(rd)
    assert [r["pipeline"] for r in rows] == ["32", "hybrid"]
    assert rows[0]["L"] == "64" and rows[1]["L"] == "4096"
    assert rows[1]["mean_ms"] == "0.600000"
    for r in rows:
        for k in sweep.HEADER[9:]:
            float(r[k])
    # a fresh write truncates
    sweep.write_csv(str(path), [rh])
    assert len(path.read_text().splitlines()) == 2


@pytest.mark.gpu
@pytest.mark.parametrize("pipeline", ["32", "hybrid", "64bit"])
def test_sweep_measures_on_the_gpu(tmp_path, pipeline):
    r = sweep.measure(pipeline, 9, warmup=1, iters=2)
    assert r["iters"] == 2 and r["mean_ms"] > 0
    assert all(r[k] >= 0 for k in PLOT_STACK)
    assert r["h2d_mean_ms"] + r["fwd_pad_ntt_mean_ms"] + r["crt_mean_ms"] > 0
    assert r["N"] >= r["L"]
    path = tmp_path / "g.csv"
    sweep.write_csv(str(path), [r])
    assert path.read_text().splitlines()[0] == REFERENCE_HEADER


def test_measured_product_is_checked():
    """measure() checks the last product by residues before it reports."""
    a = np.array([3, 1], dtype=np.uint32)
    b = np.array([5, 2], dtype=np.uint32)
    c = np.array([15, 11, 2, 0], dtype=np.uint32)
    assert sweep.product_ok(a, b, c)
    c[1] ^= 1
    assert not sweep.product_ok(a, b, c)


def test_command_line_with_a_stubbed_measurement(tmp_path, monkeypatch, capsys):
    """main(): L list parsing, sizes a pipeline cannot reach reported and
    skipped, rows appended under one header."""
    def fake_measure(pipeline, L_arg, warmup, iters):
        if L_arg == 30:
            return None
        return sweep.make_row(pipeline, L_arg, sweep.resolve_limbs(L_arg).bit_length() + 1,
                              warmup, [1.0] * iters, [stage(*[0.1] * 6)] * iters, {}, {})
    monkeypatch.setattr(sweep, "measure", fake_measure)
    path = tmp_path / "cli.csv"
    sweep.main(["--pipeline", "64bit", "--L", "6,7,30", "--iters", "2", "--csv", str(path)])
    sweep.main(["--pipeline", "32", "--L", "8", "--iters", "1", "--csv", str(path), "--append"])
    out = capsys.readouterr().out
    assert "L_arg=30: beyond" in out
    lines = path.read_text().splitlines()
    assert lines[0] == REFERENCE_HEADER and len(lines) == 4
    with open(path, newline="") as f:
        rows = list(csv.DictReader(f))
    assert [(r["pipeline"], r["L"], r["iters"]) for r in rows] == [
        ("64bit", "64", "2"), ("64bit", "128", "2"), ("32", "256", "1")]
