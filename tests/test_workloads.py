"""The seeded operand mixes of the batched and served forms (host only)."""
import numpy as np

from birdwing_b200 import workloads


def test_batch_sizes_follow_the_mix():
    s = workloads.batch_sizes(4096, seed=3)
    assert len(s) == 4096
    paths = [p for p, _, _ in s]
    assert paths.count(32) == 2048 and paths.count(64) == 2048
    la = np.array([a for _, a, _ in s])
    lb = np.array([b for _, _, b in s])
    assert la.min() >= (1 << 12) // 32 and la.max() <= (1 << 20) // 32
    assert (lb <= la).all() and (lb * 8 + 1 >= la).all()
    # log-uniform: about a quarter of the first operands in each quarter of
    # the log range (2^12..2^14, .., 2^18..2^20 bits)
    q = np.histogram(np.log2(la * 32.0), bins=[12, 14, 16, 18, 20.01])[0]
    assert (abs(q - 1024) < 150).all(), q
    assert s == workloads.batch_sizes(4096, seed=3)


def test_batch_mix_operands_have_top_bit():
    mix = workloads.batch_mix(16, seed=1)
    for p, a, b in mix:
        assert a.dtype == np.uint32 and b.dtype == np.uint32
        assert a[-1] >> 31 == 1 and b[-1] >> 31 == 1


def test_serving_sizes():
    s = workloads.serving_sizes(5000, seed=5)
    sq = sum(1 for _, _, q in s if q)
    assert 850 < sq < 1150
    for la, lb, q in s:
        assert 1 <= lb <= la <= (1 << 24) // 32
        if q:
            assert la == lb
