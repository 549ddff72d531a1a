// bw_noalloc.cu -- Garner reconstruction + carry propagation that allocates
// no device memory (bw_garner_carry_noalloc in birdwing.h).
//
// Who needs it: callers that cannot call cudaMalloc/cudaFree.  Some host
// programs hand all device memory to their own pooled allocator up front, so a
// library allocation fails or steals from the pool; others must not let a
// library call synchronise the whole device (cudaFree does), for example a
// serving loop that keeps other streams busy.  Such callers already own the
// residue arrays and the output buffer; this entry point needs nothing else
// from them.
//
// The carry look-back needs a little scratch (a tile ticket, an error word and
// one 20-byte record per 2048-word tile).  It lives in the file-scope device
// array below, of fixed size, which every GPU that loads the library keeps
// until the process exits.  In host code the name `g_noalloc_scratch` is only
// a host-side stand-in for the symbol, never a device address: its device
// address is looked up once per device with cudaGetSymbolAddress and that
// pointer is what the kernel receives.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/birdwing.h"
#include "bw_host.h"
#include "bw_kernels.cuh"

using namespace bw;

namespace {

// Scratch layout: [0,16) ticket counter, [16,20) error word, [32, 32 + 16 t)
// carry-word records, then t status words, for t <= BW_NOALLOC_MAX_TILES.
constexpr size_t kScratchBytes = 32 + (size_t)BW_NOALLOC_MAX_TILES * 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up on the
// first call for that device.
int scratch_for_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return bw_fail(BW_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return bw_fail(BW_EINVAL, "device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return bw_fail(BW_ECUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return BW_OK;
}

using u128 = unsigned __int128;
uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }
uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}
uint64_t invmod(uint64_t a, uint64_t p) { return powmod(a % p, p - 2, p); }
uint64_t companion(uint64_t w, uint64_t p, int bits) {
    return bits == 64 ? (uint64_t)(((u128)w << 64) / p) : (uint64_t)((w << 32) / p);
}
uint64_t neg_inv(uint64_t p, int bits) {
    uint64_t x = 1;
    for (int i = 0; i < 7; ++i) x *= 2 - p * x;
    const uint64_t m = bits == 64 ? ~0ull : 0xffffffffull;
    return (0 - x) & m;
}

// The constants the Garner + carry kernel reads (no twiddle tables).
template <class Ar>
void garner_constants(int path, int K, int log_n, PlanDev<Ar>& pd) {
    using T = typename Ar::T;
    const int bits = Ar::BITS;
    const uint64_t* P = bw_path_primes(path);
    memset(&pd, 0, sizeof pd);
    for (int k = 0; k < kMaxPrimes; ++k) {
        const uint64_t p = P[k < K ? k : 0];
        auto& pr = pd.pr[k];
        pr.ar.p = (T)p;
        pr.ar.p2 = (T)(2 * p);
        pr.ar.pinv = (T)neg_inv(p, bits);
        if constexpr (sizeof(T) == 8) {
            pr.ar.c = (uint32_t)(p >> 32);
            pr.ar.c3 = 3u * pr.ar.c;
            pr.ar.p3 = 3 * p;
            pr.ar.p4 = 4 * p;
            const u128 mu = (~(u128)0) / p;
            pr.ar.mu_lo = (uint64_t)mu;
            pr.ar.mu_hi = (uint32_t)(mu >> 64);
            pr.ar.oneq = (uint64_t)(((u128)1 << 64) / p);
        }
        pr.one_q = (T)companion(1, p, bits);
    }
    auto& g = pd.gar;
    g.p0 = P[0];
    g.inv1 = (T)invmod(P[0] % P[1], P[1]);
    g.inv1q = (T)companion(g.inv1, P[1], bits);
    g.p0m2 = (T)(P[0] % P[2]);
    g.p0m2q = (T)companion(g.p0m2, P[2], bits);
    g.inv2 = (T)invmod(mulmod(P[0] % P[2], P[1] % P[2], P[2]), P[2]);
    g.inv2q = (T)companion(g.inv2, P[2], bits);
    pd.K = K;
    pd.log_n = log_n;
}

template <class Ar, bool SPLIT16>
int run(int path, int K, const void* residues, size_t n, int log_n, uint32_t* out,
        size_t out_words, cudaStream_t s) {
    using T = typename Ar::T;
    const size_t NL = n / (SPLIT16 ? 2 : 1);
    // one word beyond the coefficients can hold the final carry
    const size_t words = std::max(NL, std::min(out_words, NL + 1));
    const size_t ntiles = (words + kCarryTileWords - 1) / kCarryTileWords;
    if (ntiles > (size_t)BW_NOALLOC_MAX_TILES)
        return bw_fail(BW_ESIZE,
                       "bw_garner_carry_noalloc: %zu output words need %zu carry tiles, the "
                       "fixed scratch holds %d (at most %d words)",
                       words, ntiles, BW_NOALLOC_MAX_TILES, BW_NOALLOC_MAX_TILES * kCarryTileWords);
    void* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    unsigned char* sb = static_cast<unsigned char*>(base);
    // the array keeps the previous call's contents: clear the ticket, the
    // error word and the records this call uses (epoch 1 is then fresh)
    const size_t used = 32 + ntiles * 20;
    cudaError_t e = cudaMemsetAsync(sb, 0, used, s);
    if (e != cudaSuccess) return bw_fail(BW_ECUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    PlanDev<Ar> pd;
    garner_constants<Ar>(path, K, log_n, pd);
    k_garner_carry<Ar, SPLIT16><<<(unsigned)ntiles, kCarryThreads, 0, s>>>(
        pd, static_cast<const T*>(residues), out, out_words, NL,
        reinterpret_cast<CarryState*>(sb), reinterpret_cast<uint4*>(sb + 32),
        reinterpret_cast<uint32_t*>(sb + 32 + ntiles * 16), 1u, 1u,
        reinterpret_cast<uint32_t*>(sb + 16), 1 << 22);
    e = cudaGetLastError();
    if (e != cudaSuccess) return bw_fail(BW_ECUDA, "launch: %s", cudaGetErrorString(e));
    uint32_t err = 0;
    e = cudaMemcpyAsync(&err, sb + 16, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bw_fail(BW_ECUDA, "sync: %s", cudaGetErrorString(e));
    if (err & 1u) return bw_fail(BW_ETIMEOUT, "carry look-back wait exceeded its bound");
    if (err) return bw_fail(BW_ECHECK, "residues do not reconstruct below the coefficient bound");
    return BW_OK;
}

}  // namespace

extern "C" int bw_garner_carry_noalloc(int path, int num_primes, const void* residues, size_t n,
                                       uint32_t* out, size_t out_words, void* stream) {
    bw_clear_error();
    if (path != BW_PATH_P32 && path != BW_PATH_P64)
        return bw_fail(BW_EINVAL, "path must be BW_PATH_P32 or BW_PATH_P64");
    const int K = num_primes == 0 ? 2 : num_primes;
    if (K < 2 || K > 3) return bw_fail(BW_EINVAL, "num_primes must be 2 or 3");
    if (!residues || !out) return bw_fail(BW_EINVAL, "NULL pointer");
    if (n < 16 || (n & (n - 1)) != 0)
        return bw_fail(BW_EINVAL, "n must be a power of two >= 16 (got %zu)", n);
    int log_n = 0;
    while (((size_t)1 << log_n) < n) ++log_n;
    if (((uintptr_t)residues & 15u) != 0)
        return bw_fail(BW_EINVAL, "residues must be 16-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The call reads the device error word back and waits for the stream,
    // which a stream under capture does not allow (either would invalidate
    // the caller's capture): refuse such a stream before touching it.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess)
        return bw_fail(BW_ECUDA, "cudaStreamIsCapturing: %s", cudaGetErrorString(e));
    if (cap != cudaStreamCaptureStatusNone)
        return bw_fail(BW_EINVAL,
                       "bw_garner_carry_noalloc waits for its stream to read the device error "
                       "word; the stream is being captured");
    if (path == BW_PATH_P64) return run<Ar64, false>(path, K, residues, n, log_n, out, out_words, s);
    return run<Ar32, true>(path, K, residues, n, log_n, out, out_words, s);
}
