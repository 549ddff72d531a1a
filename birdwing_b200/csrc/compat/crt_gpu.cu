// crt_gpu.cu -- stage-level Garner CRT with the reference's interface:
// constants and residue pointers in __constant__ memory, one thread per
// coefficient, launch on the legacy stream followed by a device sync
// (reference: src/crt_gpu.cu:10-302).  Works for any NUM_MODULI primes below
// 2^63; products are reduced with 128-bit remainders.
#include <cuda_runtime.h>

#include <cassert>

#include "crt_gpu.h"

__constant__ uint64_t c_primes[NUM_MODULI];
__constant__ uint64_t c_inv[NUM_MODULI];
__constant__ uint64_t c_mmod[NUM_MODULI][NUM_MODULI];
__constant__ TestDataTypeUint* c_res[NUM_MODULI];

namespace {

__device__ __forceinline__ uint64_t mm(uint64_t a, uint64_t b, uint64_t p) {
    return (uint64_t)(((unsigned __int128)a * b) % p);
}

// mixed-radix digits k_j of the residues at index i, then
// x = sum k_j (p_0 ... p_{j-1}) accumulated in `words` 64-bit words
template <int WORDS>
__device__ void garner_at(size_t i, uint64_t (&x)[WORDS]) {
    uint64_t xm[NUM_MODULI];  // x mod p_k of the partial sum
    for (int k = 0; k < NUM_MODULI; ++k) xm[k] = 0;
    uint64_t M[WORDS];  // running product p_0 ... p_{j-1}
    for (int w = 0; w < WORDS; ++w) {
        x[w] = 0;
        M[w] = w == 0 ? 1 : 0;
    }
    for (int j = 0; j < NUM_MODULI; ++j) {
        const uint64_t p = c_primes[j];
        const uint64_t r = (uint64_t)c_res[j][i] % p;
        const uint64_t t = r >= xm[j] ? r - xm[j] : r + p - xm[j];
        const uint64_t kj = mm(t, c_inv[j], p);
        for (int k = j + 1; k < NUM_MODULI; ++k) {
            const uint64_t pk = c_primes[k];
            uint64_t v = xm[k] + mm(c_mmod[j][k], kj, pk);
            xm[k] = v >= pk ? v - pk : v;
        }
        unsigned __int128 cy = 0;
        for (int w = 0; w < WORDS; ++w) {  // x += M * kj
            const unsigned __int128 s = (unsigned __int128)M[w] * kj + x[w] + cy;
            x[w] = (uint64_t)s;
            cy = s >> 64;
        }
        cy = 0;
        for (int w = 0; w < WORDS; ++w) {  // M *= p
            const unsigned __int128 s = (unsigned __int128)M[w] * p + cy;
            M[w] = (uint64_t)s;
            cy = s >> 64;
        }
    }
}

__global__ void crt2_kernel(uint64_t* __restrict__ hi, uint64_t* __restrict__ lo, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint64_t x[2];
    garner_at<2>((size_t)i, x);
    lo[i] = x[0];
    hi[i] = x[1];
}

#if defined(NATIVE_HOST_LIMBS)
__global__ void crt3_kernel(uint64_t* __restrict__ lo, uint64_t* __restrict__ mid,
                            uint32_t* __restrict__ hi, int N) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    uint64_t x[3];
    garner_at<3>((size_t)i, x);
    lo[i] = x[0];
    mid[i] = x[1];
    hi[i] = (uint32_t)x[2];
}
#endif

}  // namespace

CRTGarnerParams compute_garner_params(const vector<TestDataTypeUint>& primes) {
    assert(primes.size() == NUM_MODULI);
    CRTGarnerParams g{};
    for (int i = 0; i < NUM_MODULI; ++i) {
        const uint64_t p = primes[i];
        g.primes[i] = p;
        // (p_0 ... p_{k-1}) mod p for every k, by repeated modular products
        uint64_t prefix = 1 % p;
        for (int k = 0; k < NUM_MODULI; ++k) {
            g.M_mod_table[k][i] = prefix;
            prefix = (uint64_t)((unsigned __int128)prefix * ((uint64_t)primes[k] % p) % p);
        }
        g.prefix_M[i] = g.M_mod_table[i][i];
        g.inv[i] = i == 0 ? 1 : modinv_u64(g.prefix_M[i], p);
        g.barrett_m[i] = LIMB_BITS == 32 ? (uint64_t)(((unsigned __int128)1 << 64) / p) : 0;
    }
    return g;
}

void upload_garner_params(const CRTGarnerParams& params) {
    cudaMemcpyToSymbol(c_primes, params.primes, sizeof params.primes);
    cudaMemcpyToSymbol(c_inv, params.inv, sizeof params.inv);
    cudaMemcpyToSymbol(c_mmod, params.M_mod_table, sizeof params.M_mod_table);
}

void upload_residue_ptrs(const vector<TestDataTypeUint*>& c_dev) {
    TestDataTypeUint* p[NUM_MODULI];
    for (int j = 0; j < NUM_MODULI; ++j) p[j] = c_dev[j];
    cudaMemcpyToSymbol(c_res, p, sizeof p);
}

void crt_combine_gpu(uint64_t* d_C_hi, uint64_t* d_C_lo, int N) {
    if (N <= 0) return;
    crt2_kernel<<<(N + 255) / 256, 256>>>(d_C_hi, d_C_lo, N);
    cudaDeviceSynchronize();
}

#if defined(NATIVE_HOST_LIMBS)
void crt_combine_gpu_u160(uint64_t* d_C_lo, uint64_t* d_C_mid, uint32_t* d_C_hi, int N) {
    if (N <= 0) return;
    crt3_kernel<<<(N + 255) / 256, 256>>>(d_C_lo, d_C_mid, d_C_hi, N);
    cudaDeviceSynchronize();
}
#endif
