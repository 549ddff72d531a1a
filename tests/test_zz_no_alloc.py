"""bw_garner_carry_noalloc: the Garner + carry stage for callers that cannot
allocate device memory (a program whose pool allocator owns all of it, or a
loop that cannot let cudaFree synchronise the device).  Its output must equal
the regular entry point's product, bit for bit, on two calls in a row (the
calls share one fixed scratch array), and a call must leave the device's free
memory unchanged.  Kept in its own file, collected last."""
import ctypes

import numpy as np
import pytest

import birdwing_b200 as bw
from oracle import gmp_ref, oracle

pytestmark = pytest.mark.gpu


def residues_of(a, b, path, K, n):
    """Residues of the cyclic convolution per prime (oracle, CPU)."""
    per = 2 if path == 32 else 1
    ca = a.view(np.uint16) if per == 2 else a
    cb = b.view(np.uint16) if per == 2 else b
    primes, roots, logs = oracle.path_basis(path)
    out = []
    for k in range(K):
        w = oracle.lib.oracle_root_for(primes[k], roots[k], logs[k], n.bit_length() - 1)
        out.append(oracle.conv_mod([int(x) for x in ca], [int(x) for x in cb], primes[k], w, n))
    dt = np.uint64 if path == 64 else np.uint32
    return np.concatenate([r.astype(dt) for r in out])


@pytest.mark.parametrize("path,K,la,lb", [(64, 2, 3000, 2100), (64, 3, 777, 4096),
                                          (32, 3, 2048, 2048), (32, 2, 1500, 999)])
def test_noalloc_matches_multiply_twice(path, K, la, lb):
    import torch
    rng = np.random.default_rng(la * 7 + lb)
    a = rng.integers(0, 1 << 32, la, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 1 << 32, lb, dtype=np.uint64).astype(np.uint32)
    with bw.Plan(la, lb, path, K) as p, bw.Context(p) as c:
        want = c.multiply(a, b)
        n = p.N
    assert (want == gmp_ref.mul(a, b)).all()
    res = residues_of(a, b, path, K, n)
    d_res = torch.from_numpy(res.view(np.int64 if path == 64 else np.int32)).cuda()
    for call in range(2):
        d_out = torch.full((la + lb,), -1, dtype=torch.int32, device="cuda")
        rc = bw.lib.bw_garner_carry_noalloc(path, K, ctypes.c_void_p(d_res.data_ptr()), n,
                                            ctypes.c_void_p(d_out.data_ptr()), la + lb, None)
        assert rc == 0, bw._lib.last_error()
        got = d_out.cpu().numpy().view(np.uint32)
        assert (got == want).all(), f"call {call}"


def test_noalloc_final_carry_word_and_no_allocation():
    # the convolution fills the transform (la + lb = n): out_words = n + 1
    # asks for the final-carry word, which is zero for a product of la + lb
    # words; a call after the first allocates nothing on the device
    import torch
    la = lb = 2048
    rng = np.random.default_rng(99)
    a = rng.integers(0, 1 << 32, la, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 1 << 32, lb, dtype=np.uint64).astype(np.uint32)
    a[:] = 0xFFFFFFFF
    with bw.Plan(la, lb, 64, 2) as p, bw.Context(p) as c:
        want = c.multiply(a, b)
        n = p.N
    assert n == la + lb
    res = residues_of(a, b, 64, 2, n)
    d_res = torch.from_numpy(res.view(np.int64)).cuda()
    d_out = torch.full((n + 1,), -1, dtype=torch.int32, device="cuda")
    args = (64, 2, ctypes.c_void_p(d_res.data_ptr()), n, ctypes.c_void_p(d_out.data_ptr()),
            n + 1, None)
    assert bw.lib.bw_garner_carry_noalloc(*args) == 0, bw._lib.last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    assert bw.lib.bw_garner_carry_noalloc(*args) == 0, bw._lib.last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    got = d_out.cpu().numpy().view(np.uint32)
    assert (got[:n] == want).all() and got[n] == 0


def test_noalloc_refuses_capturing_stream():
    # the call waits for its stream, which a capture does not allow: it must
    # refuse the stream before enqueueing anything, leaving the capture valid
    import torch
    d_res = torch.zeros(64, dtype=torch.int64, device="cuda")
    d_out = torch.zeros(32, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        d_out.add_(1)                       # warm the op up before capture
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            d_out.add_(1)
            rc = bw.lib.bw_garner_carry_noalloc(64, 2, ctypes.c_void_p(d_res.data_ptr()), 32,
                                                ctypes.c_void_p(d_out.data_ptr()), 32,
                                                ctypes.c_void_p(s.cuda_stream))
    assert rc == -1 and "captured" in bw._lib.last_error()
    g.replay()                              # the captured add_ alone
    torch.cuda.synchronize()
    assert int(d_out[0]) == 2


def test_noalloc_rejects_oversize():
    big = (1 << 26) * 2048 * 2  # n beyond the fixed scratch
    rc = bw.lib.bw_garner_carry_noalloc(64, 2, ctypes.c_void_p(16), big, ctypes.c_void_p(16), 8,
                                        None)
    assert rc == -6 and "scratch" in bw._lib.last_error()
