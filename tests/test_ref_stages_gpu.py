"""Parity with the reference's own stage kernels, run on the GPU: its carry
kernels (src/carry_prop.cu with the host escape loop of src/gpu_ntt.cu) on
libbirdwing's CRT coefficients must give libbirdwing's product, and its
crt_combine_gpu (src/crt_gpu.cu) on residues of the same convolution must
give libbirdwing's coefficients.  Both built with LIMB_BITS=64 (u32 limbs,
two 64-bit primes), the configuration of the 64-bit path with K = 2."""
import ctypes
import os

import numpy as np
import pytest

import birdwing_b200 as bw
from oracle import oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_stage_hybrid.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libref_stage_hybrid.so not built")
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    lib.ref_crt_combine_hybrid.argtypes = [ctypes.c_uint64, ctypes.c_uint64, P, P, ctypes.c_int,
                                           P, P]
    lib.ref_carry_hybrid.argtypes = [P, P, ctypes.c_size_t, P]
    return lib


@pytest.mark.parametrize("la,lb", [(5, 3), (1000, 777), (4096, 4096), (30000, 12345)])
def test_reference_carry_on_our_coefficients(ref, la, lb):
    import torch
    rng = np.random.default_rng(la + lb)
    a = rng.integers(0, 1 << 32, la, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 1 << 32, lb, dtype=np.uint64).astype(np.uint32)
    with bw.Plan(la, lb, 64, 2) as p, bw.Context(p) as c:
        prod = c.multiply(a, b)
        n = p.N
        words = np.empty(3 * n, dtype=np.uint32)
        assert bw.lib.bw_multiply_coeffs(c._h, a.ctypes.data, la, b.ctypes.data, lb,
                                         words.ctypes.data, words.size) == 0
    w = words.reshape(n, 3).astype(np.uint64)
    lo = (w[:, 0] | (w[:, 1] << np.uint64(32))).astype(np.uint64)
    hi = w[:, 2].copy()
    d_hi = torch.from_numpy(hi.view(np.int64)).cuda()
    d_lo = torch.from_numpy(lo.view(np.int64)).cuda()
    d_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    assert ref.ref_carry_hybrid(d_hi.data_ptr(), d_lo.data_ptr(), n, d_out.data_ptr()) == 0
    got = d_out.cpu().numpy().view(np.uint32)
    m = min(n, la + lb)
    assert (got[:m] == prod[:m]).all()


@pytest.mark.parametrize("la,lb", [(7, 9), (2048, 1000)])
def test_reference_garner_on_same_residues(ref, la, lb):
    import torch
    rng = np.random.default_rng(3 * la + lb)
    a = rng.integers(0, 1 << 32, la, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, 1 << 32, lb, dtype=np.uint64).astype(np.uint32)
    with bw.Plan(la, lb, 64, 2) as p, bw.Context(p) as c:
        coeffs = c.coeffs(a, b)
        n = p.N
    primes, roots, logs = oracle.path_basis(64)
    res = []
    for k in range(2):
        wk = oracle.lib.oracle_root_for(primes[k], roots[k], logs[k], n.bit_length() - 1)
        res.append(oracle.conv_mod([int(x) for x in a], [int(x) for x in b], primes[k], wk, n))
    d0 = torch.from_numpy(res[0].view(np.int64)).cuda()
    d1 = torch.from_numpy(res[1].view(np.int64)).cuda()
    d_hi = torch.zeros(n, dtype=torch.int64, device="cuda")
    d_lo = torch.zeros(n, dtype=torch.int64, device="cuda")
    assert ref.ref_crt_combine_hybrid(primes[0], primes[1], d0.data_ptr(), d1.data_ptr(), n,
                                      d_hi.data_ptr(), d_lo.data_ptr()) == 0
    hi = d_hi.cpu().numpy().view(np.uint64)
    lo = d_lo.cpu().numpy().view(np.uint64)
    ref_vals = [int(h) << 64 | int(l) for h, l in zip(hi, lo)]
    assert ref_vals == coeffs
