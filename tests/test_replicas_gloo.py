"""Multi-process host logic of bench.py on CPU (gloo, world size 2): products
are independent, so N ranks run N replicas with no collective on the data
path; the only cross-rank steps are the barrier, the max over ranks of the
timed region and the sum of counts.  Also: the reference arm prints on rank 0
only and every other rank exits quietly."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        # rank r's timed region took 10 * (r + 1) ms for 4 * (r + 1) products
        t_ms, done = bench.reduce_over_ranks([10.0 * (rank + 1), 4.0 * (rank + 1)],
                                             ["max", "sum"])
        value = bench.job_throughput(4, world, t_ms)
        dist.barrier()
        q.put((rank, t_ms, done, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, t_ms, done, value in res:
        assert t_ms == 20.0            # the slowest rank
        assert done == 12.0            # 4 + 8
        assert value == pytest.approx(2 * 4 / 0.020)


def test_single_process_reduction_is_identity():
    import bench
    assert bench.reduce_over_ranks([3.5, 2.0], ["max", "sum"]) == [3.5, 2.0]
    assert bench.job_throughput(10, 1, 5.0) == pytest.approx(2000.0)


def test_reference_arm_prints_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    args = bench.parse_args_list(["--impl", "reference", "--config", "1", "--steps", "1",
                                  "--warmup", "0"])
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    assert buf.getvalue() == ""


def test_reference_arm_line_on_rank_zero(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "0")
    args = bench.parse_args_list(["--impl", "reference", "--config", "1", "--steps", "1",
                                  "--warmup", "0"])
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    line = json.loads(buf.getvalue())
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port"


def test_bench_configs_come_from_the_shared_table():
    """Plain configurations name the reference's algorithm (path, primes) for
    the oracle and the CPU baseline; the library's plan comes from the same
    table (birdwing_b200.workloads.PLAIN) that the full-size parity tests
    build their plans from."""
    import bench
    from birdwing_b200 import workloads
    assert set(bench.CONFIGS) == set(workloads.PLAIN)
    for name, w in workloads.PLAIN.items():
        la, lb, path, K, square, desc = bench.CONFIGS[name]
        assert (la, lb, square) == (w["words_a"], w["words_b"], w["square"])
        assert (path, K) == w["ref"] and K in (2, 3) and path in (32, 64)
        assert w["plan"][1] in (0, 2, 3) and w["literal"][1] in (2, 3)
        assert set(w["expect"]) <= {"path", "coeff_bits", "num_primes", "log_n", "log_cols"}
        assert workloads.plain_plan_args(name)[:2] == (la, lb)
        assert "reference algorithm" in bench.ref_algorithm(name)
    mb = bench.model_bytes(1 << 23, 1 << 23, 1 << 23, 3, 8, False)
    assert sum(mb.values()) == 12 * 3 * (1 << 23) * 8 + 4 * (2 << 23) * 2
    # the fixed model of the 2^28-bit workload: K = 2, n = 2^24, w = 8
    fixed, K, n, w = bench.fixed_model("2")
    assert (K, n, w) == (2, 1 << 24, 8)
    assert fixed == 12 * 2 * (1 << 24) * 8 + 4 * (2 << 23) * 2
    info = {"num_primes": 3, "log_n": 23}
    assert bench.plan_butterflies(info, False) == 3 * 3 * (1 << 22) * 23
