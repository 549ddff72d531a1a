// bw_probe.cu -- integer-pipe ceiling of the transforms' butterflies
// (bw_butterfly_rate in birdwing.h).
//
// The product's NTT kernels are bound by integer instruction issue, not by
// HBM, so their second roofline is the butterfly rate the SMs can sustain when
// nothing but butterflies runs.  This kernel measures it with the very
// butterflies the transforms use (Ar32 / Ar64 ct and gs from bw_arith.cuh):
// every thread keeps 16 residues in registers and applies, per iteration, two
// radix-16 forward rounds and one radix-16 inverse round (96 butterflies, the
// 2:1 mix of a product's forward and inverse transforms), with no memory
// traffic in the loop.  The reference has no counterpart: its transforms are
// the absent GPU-NTT library's (src/gpu_ntt.cu:577-581).
#include <cuda_runtime.h>

#include "../../include/birdwing.h"
#include "bw_host.h"
#include "bw_kernels.cuh"

using namespace bw;

namespace {

using u128 = unsigned __int128;

template <class Ar>
struct ProbeArgs {
    Ar ar;
    Tw<typename Ar::T> w[4];
};

template <class Ar>
__global__ void __launch_bounds__(256)
k_bfly_rate(const ProbeArgs<Ar> P, int iters, typename Ar::T* out) {
    using T = typename Ar::T;
    const Ar ar = P.ar;
    T x[16];
    const uint64_t seed = (uint64_t)(blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B97F4A7C15ull;
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = (T)((seed + k * 0x632BE59BD9B4E019ull) >> 7) % ar.p;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                const int h = 8 >> l;
                const Tw<T> w = P.w[l];
#pragma unroll
                for (int q = 0; q < (1 << l); ++q)
#pragma unroll
                    for (int u = 0; u < h; ++u) ar.ct(x[(q << (4 - l)) + u], x[(q << (4 - l)) + u + h], w.w, w.wq);
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = ar.fwd_to_2p(x[k]);
        }
#pragma unroll
        for (int l = 3; l >= 0; --l) {
            const int h = 8 >> l;
            const Tw<T> w = P.w[l];
#pragma unroll
            for (int q = 0; q < (1 << l); ++q)
#pragma unroll
                for (int u = 0; u < h; ++u) ar.gs(x[(q << (4 - l)) + u], x[(q << (4 - l)) + u + h], w.w, w.wq);
        }
    }
    T acc = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) acc ^= x[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

uint64_t companion(uint64_t w, uint64_t p, int bits) {
    return bits == 64 ? (uint64_t)(((u128)w << 64) / p) : (uint64_t)((w << 32) / p);
}

template <class Ar>
int run_probe(int iters, int ctas_per_sm, float* ms, double* butterflies) {
    using T = typename Ar::T;
    constexpr bool W = sizeof(T) == 8;
    const uint64_t p = bw_path_primes(W ? BW_PATH_P64 : BW_PATH_P32)[0];
    ProbeArgs<Ar> P{};
    P.ar.p = (T)p;
    P.ar.p2 = (T)(2 * p);
    if constexpr (W) {
        P.ar.c = (uint32_t)(p >> 32);
        P.ar.c3 = 3u * P.ar.c;
        P.ar.p3 = 3 * p;
        P.ar.p4 = 4 * p;
        P.ar.oneq = (uint64_t)(((u128)1 << 64) / p);
    }
    for (int l = 0; l < 4; ++l) {
        const uint64_t w = (0x1234567u * (l + 3)) % p;
        P.w[l].w = (T)w;
        P.w[l].wq = (T)companion(w, p, Ar::BITS);
    }
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return bw_fail(BW_ECUDA, "no current CUDA device");
    const unsigned blocks = (unsigned)(sms * ctas_per_sm);
    T* out = nullptr;
    if (cudaMalloc(&out, (size_t)blocks * 256 * sizeof(T)) != cudaSuccess)
        return bw_fail(BW_ENOMEM, "butterfly probe: cudaMalloc failed");
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = BW_OK;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = bw_fail(BW_ECUDA, "stream/event creation failed");
    } else {
        k_bfly_rate<Ar><<<blocks, 256, 0, s>>>(P, 4, out);  // warm-up
        cudaEventRecord(e0, s);
        k_bfly_rate<Ar><<<blocks, 256, 0, s>>>(P, iters, out);
        cudaEventRecord(e1, s);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            rc = bw_fail(BW_ECUDA, "butterfly probe: %s", cudaGetErrorString(e));
        } else {
            cudaEventElapsedTime(ms, e0, e1);
            *butterflies = (double)blocks * 256.0 * (double)iters * 96.0;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaFree(out);
    return rc;
}

}  // namespace

extern "C" int bw_butterfly_rate(int path, int iters, int ctas_per_sm, float* ms,
                                 double* butterflies) {
    bw_clear_error();
    if (!ms || !butterflies) return bw_fail(BW_EINVAL, "NULL pointer");
    if (iters <= 0 || ctas_per_sm <= 0 || ctas_per_sm > 8)
        return bw_fail(BW_EINVAL, "iters must be positive and ctas_per_sm in 1..8");
    if (path == BW_PATH_P64) return run_probe<Ar64>(iters, ctas_per_sm, ms, butterflies);
    if (path == BW_PATH_P32) return run_probe<Ar32>(iters, ctas_per_sm, ms, butterflies);
    return bw_fail(BW_EINVAL, "path must be BW_PATH_P32 or BW_PATH_P64");
}
