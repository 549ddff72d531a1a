// bw_core.cu -- plans, contexts, kernel launches and the C ABI (birdwing.h).
//
// Lifecycle (reference: precompute_ntt / upload_ntt_precomputed /
// allocate_ntt_context / execute_ntt_multiply / cleanup_*,
// src/gpu_ntt.cu:240-1018, and the five timing buckets of docs/TIMING.md):
//   bw_plan_create  = precompute + upload: O(R + C + sqrt(n)) twiddles per
//                     prime, built on the host and copied once;
//   bw_ctx_create   = allocate: residue scratch, staging, carry state, stream;
//   bw_multiply     = execute: H2D (host mode), K1..K4 on one stream, D2H;
//   *_destroy       = cleanup.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/birdwing.h"
#include "bw_host.h"
#include "bw_internal.h"
#include "bw_kernels.cuh"

using namespace bw;

// ------------------------------------------------------------------ errors

static thread_local std::string g_last_error;

int bw_fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}
void bw_clear_error() { g_last_error.clear(); }

#define BW_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            return bw_fail(e_ == cudaErrorMemoryAllocation ? BW_ENOMEM : BW_ECUDA,      \
                           "%s failed: %s", #call, cudaGetErrorString(e_));             \
        }                                                                               \
    } while (0)

// ------------------------------------------------------------------ host math

namespace {

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
uint64_t shoup_pre(uint64_t w, uint64_t p, int bits) {
    return bits == 64 ? (uint64_t)(((u128)w << 64) / p) : (uint64_t)((((uint64_t)w) << 32) / p);
}
uint64_t neg_inv_pow2(uint64_t p, int bits) {
    uint64_t x = 1;  // Newton: x = x * (2 - p x) doubles the correct bits
    for (int i = 0; i < 7; ++i) x *= 2 - p * x;
    if (bits == 32) x &= 0xffffffffull;
    const uint64_t m = bits == 64 ? ~0ull : 0xffffffffull;
    return (0 - x) & m;
}
uint32_t bitrev_h(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) {
        r = (r << 1) | (x & 1);
        x >>= 1;
    }
    return r;
}

// Primes of the two paths with a generator of the multiplicative group.
// P64: c * 2^32 + 1, the largest such primes below 2^58 (v2(p-1) = 32): 64p
//      fits in 64 bits, so a forward transform of up to 20 stages adds its
//      butterflies' sums without reducing them (values stay below 3p (s + 1)
//      after s stages); three of them (2^174) still carry 64-bit
//      coefficients, whose convolution stays below 2^160.
// P32: primes below 2^30 with v2(p-1) = 26, 25, 24: the first two (K = 2)
//      allow transforms of 2^25 points, and their product (2^56.1) bounds
//      every product of that length (min(L_A, L_B) (2^16 - 1)^2 < p0 p1).
const uint64_t kP64[3] = {0x3ffffd500000001ull, 0x3ffffcf00000001ull, 0x3ffffa500000001ull};
const uint64_t kG64[3] = {5, 11, 7};
const uint64_t kP32[3] = {469762049ull, 167772161ull, 754974721ull};
const uint64_t kG32[3] = {3, 3, 11};
// P32 with 64-bit coefficients: the six primes below 2^30 with v2(p-1) >= 23
// and the largest residues, in ascending order (garner6_words_at relies on
// it): transforms of up to 2^23 points, and a product of 2^177 against the
// 2^150 bound of 2^22 coefficients of 64 bits (min(na, nb) 2^128).
const uint64_t kP32W[6] = {595591169ull, 645922817ull, 754974721ull,
                           880803841ull, 897581057ull, 998244353ull};
const uint64_t kG32W[6] = {3, 3, 11, 26, 3, 3};

int v2(uint64_t x) {
    int k = 0;
    while ((x & 1) == 0) {
        x >>= 1;
        ++k;
    }
    return k;
}

}  // namespace

int bw_path_max_log_n(int path, int K) {
    const uint64_t* P = path == BW_PATH_P64 ? kP64 : kP32;
    int m = 64;
    for (int k = 0; k < K; ++k) m = std::min(m, v2(P[k] - 1));
    // three-pass schedule: C <= 2^12, R, R2 <= 2^11 (larger sizes are bounded
    // by device memory, checked when the context is allocated)
    const int design = 34;
    return std::min(m, design);
}

const uint64_t* bw_path_primes(int path) { return path == BW_PATH_P64 ? kP64 : kP32; }

// The prime set of a plan and its generators: the path's own, or the six
// 32-bit primes when the 32-bit path carries 64-bit coefficients.
static const uint64_t* plan_primes(int path, bool w64) {
    return (w64 && path == BW_PATH_P32) ? kP32W : bw_path_primes(path);
}
static const uint64_t* plan_gens(int path, bool w64) {
    return (w64 && path == BW_PATH_P32) ? kG32W : path == BW_PATH_P64 ? kG64 : kG32;
}

// ------------------------------------------------------------------ plan

namespace {

template <class Ar>
struct TableBuilder {
    using T = typename Ar::T;
    std::vector<Tw<T>> host;
    // returns element offset of a new table
    // every table starts at an even entry (16 bytes for 4-byte residues), so
    // that the transforms can load its entries in pairs
    void align_even() {
        if (host.size() & 1) host.push_back(Tw<T>{0, 0});
    }
    size_t add_stage_table(uint64_t p, uint64_t root, int log_len, int bits) {
        const size_t L = (size_t)1 << log_len;
        align_even();
        const size_t off = host.size();
        host.resize(off + std::max<size_t>(L, 1));
        std::vector<uint64_t> pw(std::max<size_t>(L / 2, 1));
        pw[0] = 1;
        for (size_t j = 1; j < pw.size(); ++j) pw[j] = mulmod(pw[j - 1], root, p);
        host[off] = Tw<T>{0, 0};
        for (int s = 0; s < log_len; ++s) {
            const size_t m = (size_t)1 << s;
            for (size_t i = 0; i < m; ++i) {
                const size_t e = (L >> (s + 1)) * bitrev_h((uint32_t)i, s);
                const uint64_t w = pw[e];
                host[off + m + i] = Tw<T>{(T)w, (T)shoup_pre(w, p, bits)};
            }
        }
        return off;
    }
    size_t add_power_table(uint64_t p, uint64_t base, size_t count, uint64_t scale, int bits) {
        align_even();
        const size_t off = host.size();
        host.resize(off + count);
        uint64_t w = scale % p;
        for (size_t j = 0; j < count; ++j) {
            host[off + j] = Tw<T>{(T)w, (T)shoup_pre(w, p, bits)};
            w = mulmod(w, base, p);
        }
        return off;
    }
};

inline void set_c(Ar32& a, uint64_t p) {
    a.pinv_d = 4294967296.0 / (double)p;
    a.r32 = (uint32_t)(((uint64_t)1 << 32) % p);
    a.r32q = (uint32_t)shoup_pre(a.r32, p, 32);
    a.oneq = (uint32_t)(((uint64_t)1 << 32) / p);
}
inline void set_c(Ar64& a, uint64_t p) {
    a.c = (uint32_t)(p >> 32);
    a.c3 = 3u * a.c;
    a.p3 = 3 * p;
    a.p4 = 4 * p;
    const u128 mu = (~(u128)0) / p;  // floor(2^128 / p): p is odd
    a.mu_lo = (uint64_t)mu;
    a.mu_hi = (uint32_t)(mu >> 64);
    a.oneq = (uint64_t)(((u128)1 << 64) / p);
}

template <class Ar>
int build_tables(bw_plan* pl, PlanDev<Ar>& pd) {
    using T = typename Ar::T;
    const int bits = Ar::BITS;
    const uint64_t* P = plan_primes(pl->path, pl->w64 != 0);
    const uint64_t* Gn = plan_gens(pl->path, pl->w64 != 0);
    TableBuilder<Ar> tb;
    size_t off[kMaxPrimes][12];
    const size_t n = (size_t)1 << pl->log_n;
    // row-level twiddle length: R * C (two passes) or R2 * C (three passes)
    const int log_rr = pl->log_r2 ? pl->log_r2 : pl->log_r;
    const size_t n_row = (size_t)1 << (log_rr + pl->log_c);
    uint64_t scale_k[kMaxPrimes] = {};
    for (int k = 0; k < pl->K; ++k) {
        const uint64_t p = P[k];
        scale_k[k] = mulmod(invmod(n % p, p), powmod(2, bits, p), p);
        if (pl->small) {
            // single pass: n-point stage tables only
            const uint64_t wn = powmod(Gn[k], (p - 1) >> pl->log_n, p);
            off[k][2] = tb.add_stage_table(p, wn, pl->log_n, bits);
            off[k][3] = tb.add_stage_table(p, invmod(wn, p), pl->log_n, bits);
            continue;
        }
        const uint64_t wn = powmod(Gn[k], (p - 1) >> pl->log_n, p);  // primitive n-th root
        const uint64_t wrow = powmod(wn, n / n_row, p);               // n_row-th root
        const uint64_t wrowi = invmod(wrow, p);
        const uint64_t wr = powmod(wn, n >> pl->log_r, p);            // R-th root
        const uint64_t wc = powmod(wn, n >> pl->log_c, p);            // C-th root
        off[k][0] = tb.add_stage_table(p, wr, pl->log_r, bits);
        off[k][1] = tb.add_stage_table(p, invmod(wr, p), pl->log_r, bits);
        off[k][2] = tb.add_stage_table(p, wc, pl->log_c, bits);
        off[k][3] = tb.add_stage_table(p, invmod(wc, p), pl->log_c, bits);
        const size_t nlo = (size_t)1 << pl->lo, nhi = n_row >> pl->lo;
        const uint64_t scale = mulmod(invmod(n % p, p), powmod(2, bits, p), p);
        off[k][4] = tb.add_power_table(p, wrow, nlo, 1, bits);
        off[k][5] = tb.add_power_table(p, powmod(wrow, nlo, p), nhi, 1, bits);
        off[k][6] = tb.add_power_table(p, wrowi, nlo, 1, bits);
        off[k][7] = tb.add_power_table(p, powmod(wrowi, nlo, p), nhi, scale, bits);
        if (pl->log_r2) {
            const uint64_t wm = powmod(wn, n >> pl->log_r2, p);  // R2-th root
            off[k][8] = tb.add_stage_table(p, wm, pl->log_r2, bits);
            off[k][9] = tb.add_stage_table(p, invmod(wm, p), pl->log_r2, bits);
            const size_t olo = (size_t)1 << pl->lo_out, ohi = n >> pl->lo_out;
            off[k][10] = tb.add_power_table(p, wn, olo, 1, bits);
            off[k][11] = tb.add_power_table(p, powmod(wn, olo, p), ohi, 1, bits);
        }
    }
    pl->table_bytes = tb.host.size() * sizeof(Tw<T>);
    BW_CUDA(cudaMalloc(&pl->d_tables, pl->table_bytes));
    BW_CUDA(cudaMemcpy(pl->d_tables, tb.host.data(), pl->table_bytes, cudaMemcpyHostToDevice));
    const Tw<T>* base = reinterpret_cast<const Tw<T>*>(pl->d_tables);
    for (int k = 0; k < pl->K; ++k) {
        auto& pr = pd.pr[k];
        pr.scale = Tw<T>{(T)scale_k[k], (T)shoup_pre(scale_k[k], P[k], bits)};
        if (pl->small) {
            pr.WCf = base + off[k][2];
            pr.WCi = base + off[k][3];
            pr.ar.p = (T)P[k];
            pr.ar.p2 = (T)(2 * P[k]);
            pr.ar.pinv = (T)neg_inv_pow2(P[k], bits);
            set_c(pr.ar, P[k]);
            pr.one_q = (T)shoup_pre(1, P[k], bits);
            continue;
        }
        pr.WRf = base + off[k][0];
        pr.WRi = base + off[k][1];
        pr.WCf = base + off[k][2];
        pr.WCi = base + off[k][3];
        pr.TLf = base + off[k][4];
        pr.THf = base + off[k][5];
        pr.TLi = base + off[k][6];
        pr.THi = base + off[k][7];
        pr.WMf = pl->log_r2 ? base + off[k][8] : nullptr;
        pr.WMi = pl->log_r2 ? base + off[k][9] : nullptr;
        pr.OLf = pl->log_r2 ? base + off[k][10] : nullptr;
        pr.OHf = pl->log_r2 ? base + off[k][11] : nullptr;
        pr.ar.p = (T)P[k];
        pr.ar.p2 = (T)(2 * P[k]);
        pr.ar.pinv = (T)neg_inv_pow2(P[k], bits);
        set_c(pr.ar, P[k]);
        pr.one_q = (T)shoup_pre(1, P[k], bits);
    }
    // unused prime slots get harmless arithmetic constants
    for (int k = pl->K; k < kMaxPrimes; ++k) pd.pr[k] = pd.pr[0];
    auto& g = pd.gar;
    const uint64_t p0 = P[0], p1 = P[1], p2 = P[2];
    g.p0 = p0;
    g.inv1 = (T)invmod(p0 % p1, p1);
    g.inv1q = (T)shoup_pre(g.inv1, p1, bits);
    g.p0m2 = (T)(p0 % p2);
    g.p0m2q = (T)shoup_pre(g.p0m2, p2, bits);
    g.inv2 = (T)invmod(mulmod(p0 % p2, p1 % p2, p2), p2);
    g.inv2q = (T)shoup_pre(g.inv2, p2, bits);
    g.p01_lo = (uint64_t)((u128)p0 * p1);
    g.p01_hi = (uint64_t)(((u128)p0 * p1) >> 64);
    if (pl->K == 6) {
        for (int i = 1; i < 6; ++i)
            for (int j = 0; j < i; ++j) {
                const uint64_t v = invmod(P[j] % P[i], P[i]);
                g.inv6[i * (i - 1) / 2 + j] = Tw<T>{(T)v, (T)shoup_pre(v, P[i], bits)};
            }
    }
    pd.K = pl->K;
    pd.log_n = pl->log_n;
    pd.log_r = pl->log_r;
    pd.log_c = pl->log_c;
    pd.lo = pl->lo;
    pd.log_cb = pl->log_cb;
    pd.log_cb1 = pl->log_cb1;
    pd.tw_smem_r = pl->tw_smem_r;
    pd.log_fa = pl->log_c / 2;
    pd.log_r2 = pl->log_r2;
    pd.log_cb2 = pl->log_cb2;
    pd.lo_out = pl->lo_out;
    return BW_OK;
}

int ceil_log2(size_t x) {
    int k = 0;
    while (((size_t)1 << k) < x) ++k;
    return k;
}

}  // namespace

int bw_check_size(int path, int K, size_t la, size_t lb, int* log_n_out) {
    if (path != BW_PATH_P32 && path != BW_PATH_P64)
        return bw_fail(BW_EINVAL, "unknown path %d", path);
    if (K < 2 || K > 3) return bw_fail(BW_EINVAL, "num_primes must be 2 or 3 (got %d)", K);
    if (la == 0 || lb == 0) return bw_fail(BW_ESIZE, "operand limb count must be positive");
    const int cpw = path == BW_PATH_P32 ? 2 : 1;
    const size_t nca = la * cpw, ncb = lb * cpw;
    // n >= 16 keeps every 64-byte vector load of the Garner kernel in bounds
    const int log_n = std::max(4, ceil_log2(nca + ncb - 1));
    const int max_log = bw_path_max_log_n(path, K);
    if (log_n > max_log)
        return bw_fail(BW_ESIZE,
                       "transform length 2^%d for %zu x %zu words exceeds the %d-bit path limit "
                       "2^%d",
                       log_n, la, lb, path, max_log);
    // CRT bound: min(L_A, L_B) * (2^b - 1)^2 < p0 * p1 (the reference's bound,
    // src/ntt_limits.cpp:82-95, against the first two primes: a third prime is
    // kept redundant so that it can check the reconstruction)
    const uint64_t* P = bw_path_primes(path);
    const int cb = path == BW_PATH_P32 ? 16 : 32;
    const long double lim = (long double)P[0] * (long double)P[1];
    const long double cmax = (long double)std::min(nca, ncb) * powl(2.0L, 2 * cb);
    if (!(cmax < lim))
        return bw_fail(BW_ESIZE, "convolution coefficient bound exceeds the CRT modulus product");
    if (log_n_out) *log_n_out = log_n;
    return BW_OK;
}

// 64-bit path with 64-bit coefficients and three primes: ceil(l / 2)
// coefficients per operand; every coefficient of the product is below
// min(na, nb) 2^128, far under p0 p1 p2 (2^184.9) for any size the
// transform reaches, and all three primes carry it (none is redundant).
// On the 32-bit path (six primes, v2(p - 1) >= 23) the transform reaches 2^23
// points, 2^23-word operands; the six primes' product (2^177) bounds every
// coefficient there (min(na, nb) 2^128 <= 2^150).
int bw_check_size_w64(size_t la, size_t lb, int* log_n_out, int path = BW_PATH_P64) {
    if (la == 0 || lb == 0) return bw_fail(BW_ESIZE, "operand limb count must be positive");
    const size_t nca = (la + 1) / 2, ncb = (lb + 1) / 2;
    const int log_n = std::max(4, ceil_log2(nca + ncb - 1));
    int max_log = bw_path_max_log_n(BW_PATH_P64, 3);
    if (path == BW_PATH_P32) {
        max_log = 64;
        for (int k = 0; k < 6; ++k) max_log = std::min(max_log, v2(kP32W[k] - 1));
    }
    if (log_n > max_log)
        return bw_fail(BW_ESIZE,
                       "transform length 2^%d for %zu x %zu words exceeds the %d-bit path limit "
                       "for 64-bit coefficients 2^%d",
                       log_n, la, lb, path == BW_PATH_P32 ? 32 : 64, max_log);
    if (log_n_out) *log_n_out = log_n;
    return BW_OK;
}

// num_primes 0 on the 64-bit path: 64-bit coefficients with three primes
// (3 primes x n/2 points instead of 2 x n) where they halve the transform
// and their own transform has at least 2^19 points.  On a B200 they measured
// faster from there (2^20-word operands: 0.245 vs 0.324 ms; 2^23: 1.93 vs
// 2.58 ms); below, the three-prime Garner and fixed costs make them slower
// (2^18 words: 0.124 vs 0.100 ms).  Every product that BW_PATH_AUTO moves off
// the 32-bit path (more than 2^21 of its points) has at least 2^19 of them.
constexpr int kW64MinLogN = 19;

bool bw_w64_pays(size_t la, size_t lb) {
    int l32 = 0, l64 = 0;
    if (bw_check_size_w64(la, lb, &l64) != BW_OK) {
        bw_clear_error();
        return false;
    }
    if (bw_check_size(BW_PATH_P64, 2, la, lb, &l32) != BW_OK) {
        bw_clear_error();
        return true;
    }
    return l64 >= kW64MinLogN && l64 < l32;
}

// BW_PATH_AUTO: the 32-bit path while its transform has at most 2^24 points
// (its 32-bit butterflies are about four times cheaper than the 64-bit ones,
// which more than pays for its doubled transform length against 32-bit
// coefficients on the 64-bit path: on a B200 it measured 10-30% faster from
// 2^14- to 2^27-bit operands, equal at 2^28), the 64-bit path beyond and
// wherever the 32-bit path cannot hold the product.  Where the 64-bit path
// would use 64-bit coefficients (w64_ok: single products with num_primes 0)
// the crossover is at 2^21 points of the 32-bit path: 2^20-word operands
// measured 0.245 ms against 0.282 ms, 2^22 words 1.00 against 1.13 ms, 2^18
// words 0.124 against 0.091 ms.
constexpr int kAutoP32MaxLogN = 24;
constexpr int kAutoP32MaxLogNW64 = 21;

int bw_choose_path(int K, size_t la, size_t lb, bool w64_ok) {
    int log_n = 0;
    const int lim = w64_ok ? kAutoP32MaxLogNW64 : kAutoP32MaxLogN;
    if (bw_check_size(BW_PATH_P32, K, la, lb, &log_n) == BW_OK && log_n <= lim)
        return BW_PATH_P32;
    bw_clear_error();
    return BW_PATH_P64;
}

// Path, prime count and coefficient width of a single-product plan.
static int resolve_plan(int path, int num_primes, size_t la, size_t lb, unsigned flags,
                        int* path_out, int* K_out, bool* w64_out) {
    int K = num_primes == 0 ? 2 : num_primes;
    bool force64 = (flags & BW_PLAN_COEF64) != 0;
    if (path == BW_PATH_AUTO) {
        path = force64 ? BW_PATH_P64
                       : bw_choose_path(K < 2 || K > 3 ? 2 : K, la, lb, num_primes == 0);
        // a single product the 16-bit split leaves: 64-bit coefficients on
        // the 32-bit path (six primes) while their transform fits (n <= 2^23);
        // on a B200 they measured faster than the 64-bit path's from 2^20-word
        // operands (0.206 vs 0.213 ms; 2^21 words 0.347 vs 0.387, 2^22 0.690
        // vs 0.760, 2^23 1.356 vs 1.514 ms)
        if (!force64 && num_primes == 0 && path == BW_PATH_P64) {
            if (bw_check_size_w64(la, lb, nullptr, BW_PATH_P32) == BW_OK) {
                path = BW_PATH_P32;
                force64 = true;
            } else {
                bw_clear_error();
            }
        }
    }
    bool w64 = false;
    if (force64) {
        const int kw = path == BW_PATH_P32 ? 6 : 3;
        if (num_primes != 0 && num_primes != kw)
            return bw_fail(BW_EINVAL, "64-bit coefficients need num_primes %d (or 0) on the "
                                      "%d-bit path", kw, path == BW_PATH_P32 ? 32 : 64);
        w64 = true;
    } else if (num_primes == 0 && path == BW_PATH_P64) {
        w64 = bw_w64_pays(la, lb);
    }
    if (w64) K = path == BW_PATH_P32 ? 6 : 3;
    *path_out = path;
    *K_out = K;
    *w64_out = w64;
    return BW_OK;
}

// Streaming multiprocessors of the current device (148 on a B200), looked up
// once per device.
static unsigned sm_count() {
    static std::atomic<unsigned> cache[64];
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (dev >= 0 && dev < 64) {
        const unsigned c = cache[dev].load(std::memory_order_relaxed);
        if (c) return c;
    }
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        return 148;
    if (dev >= 0 && dev < 64) cache[dev].store((unsigned)n, std::memory_order_relaxed);
    return (unsigned)n;
}

constexpr int kTmaColsMinLogN = 20;

int bw_plan_setup(bw_plan* pl, int path, int K, int log_n, unsigned flags, int mode) {
    pl->path = path;
    pl->K = K;
    pl->log_n = log_n;
    const int w = path == BW_PATH_P64 ? 8 : 4;
    const int max_c = path == BW_PATH_P64 ? 13 : 14;
    if (mode == 1) {
        pl->small = 1;
        pl->log_c = log_n;
        pl->log_r = 0;
    } else {
        // two passes per transform while the column length fits a CTA
        // (R <= 2^13), three passes (n = R * R2 * C) beyond, or when asked for
        const bool three = (flags & BW_PLAN_THREE_PASS) || log_n > 26;
        const int want_c = (int)((flags >> 8) & 0x1f);
        if (!three) {
            // one product: a square split; a batch group (mode 0): long rows
            // (C = 2^min(12, log n - 3) on the 64-bit path) and short columns:
            // the rows keep every thread of the row pass busy even for small
            // n, and the group's grid has a product dimension to fill the SMs
            pl->log_c = mode == 0 ? std::max(std::min(max_c - 1, log_n - 3), (log_n + 1) / 2)
                                  : std::min(max_c, (log_n + 1) / 2);
            if (want_c) {
                if (want_c > max_c || want_c >= log_n || log_n - want_c > 13)
                    return bw_fail(BW_EINVAL, "BW_PLAN_LOG_COLS(%d) invalid for n = 2^%d",
                                   want_c, log_n);
                pl->log_c = want_c;
            }
            pl->log_r = log_n - pl->log_c;
        } else {
            pl->log_c = std::min(12, log_n - 2);
            if (want_c) {
                if (want_c > max_c || want_c > log_n - 2 || log_n - want_c > 22)
                    return bw_fail(BW_EINVAL, "BW_PLAN_LOG_COLS(%d) invalid for n = 2^%d",
                                   want_c, log_n);
                pl->log_c = want_c;
            }
            const int rem = log_n - pl->log_c;
            pl->log_r = (rem + 1) / 2;
            pl->log_r2 = rem - pl->log_r;
            if (pl->log_r > 11 || pl->log_r2 > 11)
                return bw_fail(BW_ESIZE, "transform length 2^%d beyond the three-pass schedule",
                               log_n);
        }
        const int log_cols_outer = pl->log_c + pl->log_r2;  // row length of the outer pass
        // column tile: 64 KiB of residues per shared-memory buffer (128 KiB
        // with BW_PLAN_WIDE_COLS: wider row segments per CTA, fewer CTAs per SM)
        const bool wide = (flags & BW_PLAN_WIDE_COLS) != 0;
        const size_t tile_bytes = wide ? 131072 : 65536;
        auto fits = [&](int cb) {
            const size_t elems = (size_t)1 << (pl->log_r + cb);
            // the forward column pass also stages the tile's 32-bit coefficients
            return w * elems <= tile_bytes && (!wide || (w + 4) * elems <= 196608);
        };
        int log_cb = 0;
        while (log_cb < log_cols_outer && fits(log_cb + 1)) ++log_cb;
        // small transforms: narrower tiles so that the column passes still
        // put two CTAs on every SM (rows keep >= 16-byte segments)
        // (single products only: a batch group has a grid dimension per product)
        const int min_cb = w == 8 ? 1 : 2;
        const unsigned sms = mode == 2 ? sm_count() : 0u;
        while (log_cb > min_cb && (2u << (log_cols_outer - log_cb)) < 2u * sms) --log_cb;
        pl->log_cb = log_cb;
        // forward column pass: its tile also stages the coefficients (16-bit
        // halves as u16 on the 32-bit path, 32-bit limbs on the 64-bit path of
        // a batch group); residues + coefficients (+ staged twiddles) within
        // 112 KiB keep two CTAs on an SM.  A single product on the 64-bit path
        // stages them inside the residue tile (one prime per CTA), so only
        // the residues count there.
        pl->tw_smem_r =
            ((flags & BW_PLAN_TW_SMEM) && ((size_t)2 * w << pl->log_r) <= 32768) ? 1 : 0;
        // 64-bit coefficients on the 32-bit path: the forward column pass
        // loops over the six primes with a u64 copy of the coefficients beside
        // the residue tile, or (BW_PLAN_K1_ONE_PRIME) runs one prime per CTA
        // and reduces the coefficients straight into its tile; the loop
        // measured 0.3-4% faster from 2^20- to 2^23-word operands
        pl->k1_pp = (path == BW_PATH_P32 && pl->w64 && mode == 2 &&
                     (flags & BW_PLAN_K1_ONE_PRIME))
                        ? 1
                        : 0;
        // operands that both fill at most half the rows (the zero pad): only
        // those rows' coefficients are staged, so the u64 copy takes half
        pl->coef_half = (path == BW_PATH_P32 && pl->w64 && mode == 2 && !pl->k1_pp &&
                         pl->zt_a && pl->zt_b)
                            ? 1
                            : 0;
        const size_t cbytes = path == BW_PATH_P32
                                  ? (pl->w64 ? (pl->k1_pp ? 0 : pl->coef_half ? 4 : 8) : 2)
                              : mode == 2         ? 0
                              : pl->w64           ? 8
                                                  : 4;
        const size_t tsb = pl->tw_smem_r ? ((size_t)2 * w << pl->log_r) : 0;
        auto fits1 = [&](int cb) {
            const size_t elems = (size_t)1 << (pl->log_r + cb);
            return w * tile_elems(elems) + cbytes * elems + tsb <= (wide ? 196608u : 114688u);
        };
        int log_cb1 = 0;
        while (log_cb1 < log_cols_outer && fits1(log_cb1 + 1)) ++log_cb1;
        while (log_cb1 > min_cb && (2u << (log_cols_outer - log_cb1)) < 2u * sms) --log_cb1;
        pl->log_cb1 = log_cb1;
        if (pl->log_r2) {
            int l2 = 0;
            while (l2 < pl->log_c && ((size_t)w << (pl->log_r2 + l2 + 1)) <= 65536) ++l2;
            pl->log_cb2 = l2;
        }
        // column stage twiddles: read through L1 by default (measured faster
        // than staging them in shared memory, which costs occupancy); staged on
        // request when they take <= 32 KiB
        // row pass rounds: radix 8 for single products on the 64-bit path with
        // rows of at most 2^12 points (its 256-thread kernel takes 64
        // registers, no spills, and fits three CTAs per SM; measured 3-8%
        // faster per product from 2^20 to 2^23 words), radix 16 elsewhere
        // (2^13-point rows take 128 KiB of shared memory: one CTA per SM)
        const bool r8_default = mode == 2 && path == BW_PATH_P64 && pl->log_c <= 12;
        // column passes: radix 8 on request (single products on the 64-bit path)
        pl->rlog_col = ((flags & BW_PLAN_COL_RADIX8) && mode == 2 && path == BW_PATH_P64) ? 3 : 4;
        pl->rlog_row = (flags & BW_PLAN_RADIX8)    ? 3
                       : (flags & BW_PLAN_RADIX16) ? 4
                       : r8_default                ? 3
                                                   : 4;
        // inverse column tiles by tensor copies: single products with two
        // passes, from 2^20 points unless forced either way (a box is at most
        // 256 columns wide and 16 bytes or more).  Measured at 2^23 words:
        // the inverse pass 0.246 -> 0.231 ms (64-bit coefficients), 0.378 ->
        // 0.348 ms (32-bit path); at 2^17 points 0.016 -> 0.018 ms.
        const bool tma_want = (flags & BW_PLAN_TMA_COLS) ||
                              (!(flags & BW_PLAN_NO_TMA_COLS) && log_n >= kTmaColsMinLogN);
        pl->tma_cols = (tma_want && mode == 2 && pl->log_r2 == 0 && !pl->tw_smem_r &&
                        pl->log_cb <= 8 && (w << pl->log_cb) >= 16)
                           ? 1
                           : 0;
        pl->shfl_rows = ((flags & BW_PLAN_SHFL_ROWS) && mode == 2 && path == BW_PATH_P32 &&
                         pl->log_c == 12 && pl->rlog_row == 4)
                            ? 1
                            : 0;
        pl->lo = ((pl->log_r2 ? pl->log_r2 : pl->log_r) + pl->log_c + 1) / 2;
        pl->lo_out = (log_n + 1) / 2;
    }
    for (int k = 0; k < K; ++k) pl->primes[k] = plan_primes(path, pl->w64 != 0)[k];
    cudaGetDevice(&pl->device);
    const int rc =
        path == BW_PATH_P64 ? build_tables<Ar64>(pl, pl->pd64) : build_tables<Ar32>(pl, pl->pd32);
    if (rc && pl->d_tables) {
        cudaFree(pl->d_tables);
        pl->d_tables = nullptr;
    }
    return rc;
}

extern "C" int bw_plan_create(bw_plan** out, int path, size_t la, size_t lb, int num_primes,
                              unsigned flags) {
    bw_clear_error();
    if (!out) return bw_fail(BW_EINVAL, "out is NULL");
    *out = nullptr;
    int K = 0;
    bool w64 = false;
    int rc = resolve_plan(path, num_primes, la, lb, flags, &path, &K, &w64);
    if (rc) return rc;
    int log_n = 0;
    rc = w64 ? bw_check_size_w64(la, lb, &log_n, path) : bw_check_size(path, K, la, lb, &log_n);
    if (rc) return rc;
    bw_plan* pl = new bw_plan();
    pl->la = la;
    pl->lb = lb;
    pl->w64 = w64 ? 1 : 0;
    const int cpw = path == BW_PATH_P32 ? 2 : 1;
    pl->nca = w64 ? (la + 1) / 2 : la * cpw;
    pl->ncb = w64 ? (lb + 1) / 2 : lb * cpw;
    const size_t half = ((size_t)1 << log_n) / 2;
    pl->zt_a = pl->nca <= half;
    pl->zt_b = pl->ncb <= half;
    rc = bw_plan_setup(pl, path, K, log_n, flags, 2);
    if (rc) {
        delete pl;
        return rc;
    }
    pl->order = new bw_stage_order();
    *out = pl;
    return BW_OK;
}

extern "C" int bw_plan_destroy(bw_plan* pl) {
    if (!pl) return BW_OK;
    if (pl->d_tables) cudaFree(pl->d_tables);
    delete pl->order;
    delete pl;
    return BW_OK;
}

// Output words the plan's n coefficients cover: n/2 (16-bit), n (32-bit) or
// 2n (64-bit coefficients).
static size_t coef_words(const bw_plan* pl) {
    const size_t n = (size_t)1 << pl->log_n;
    return pl->w64 ? 2 * n : pl->path == BW_PATH_P32 ? n / 2 : n;
}

static size_t ctx_bytes(const bw_plan* pl) {
    const size_t n = (size_t)1 << pl->log_n;
    const int w = pl->path == BW_PATH_P64 ? 8 : 4;
    const size_t nl = std::max(coef_words(pl), pl->la + pl->lb);
    const size_t ntiles = (nl + kCarryTileWords - 1) / kCarryTileWords;
    return 2 * (size_t)pl->K * n * w + (pl->la + pl->lb) * 4 * 2 + 64 + ntiles * 20;
}

extern "C" int bw_plan_get_info(const bw_plan* pl, bw_plan_info* o) {
    if (!pl || !o) return bw_fail(BW_EINVAL, "NULL argument");
    memset(o, 0, sizeof *o);
    o->path = pl->path;
    o->num_primes = pl->K;
    o->log_n = pl->log_n;
    o->log_rows = pl->log_r;
    o->log_cols = pl->log_c;
    o->coeff_bits = pl->w64 ? 64 : pl->path == BW_PATH_P32 ? 16 : 32;
    o->la = pl->la;
    o->lb = pl->lb;
    o->lc = pl->la + pl->lb;
    o->plan_device_bytes = pl->table_bytes;
    o->ctx_device_bytes = ctx_bytes(pl);
    for (int k = 0; k < kMaxPrimes; ++k) o->primes[k] = k < pl->K ? pl->primes[k] : 0;
    return BW_OK;
}

// ------------------------------------------------------------------ context

// Most chunks a host copy is split into (see bw_ctx::copy_chunks).
constexpr int kMaxCopyChunks = 16;

struct bw_ctx {
    const bw_plan* plan = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    void* d_res_a = nullptr;
    void* d_res_b = nullptr;
    uint32_t* d_in = nullptr;   // staging: a then b
    uint32_t* d_out = nullptr;  // staging: product
    unsigned char* d_state = nullptr;
    size_t state_bytes = 0;
    CarryState* cst = nullptr;
    uint32_t* err = nullptr;
    uint4* rec_x = nullptr;
    uint32_t* rec_s = nullptr;
    size_t ntiles = 0;
    // look-back record tag of the last product.  Direct launches use 2, 3, ..;
    // the replayable graph clears the records and always uses 1.
    uint32_t epoch = 1;
    bool capturing = false;
    cudaGraphExec_t gexec = nullptr;  // device-pointer product, replayed while
    const void* g_a = nullptr;        // the pointers stay the same
    const void* g_b = nullptr;
    const void* g_out = nullptr;
    bool g_sq = false;
    uint32_t* h_err = nullptr;  // pinned
    cudaEvent_t ev[8] = {};
    cudaEvent_t stage_ev[3] = {};  // ends of copy-in, kernels, copy-out (stage order)
    bool counted = false;          // included in the plan's live contexts
    // host copies split into chunks that overlap the first and last kernels
    // (created on first use): copy-in on in_stream, copy-out on out_stream
    int copy_chunks = 0;           // 0: automatic, 1: whole copies on the stream
    cudaStream_t in_stream = nullptr, out_stream = nullptr;
    cudaEvent_t in_ev[kMaxCopyChunks] = {}, out_ev[kMaxCopyChunks] = {};
    cudaEvent_t ready_ev = nullptr, out_done_ev = nullptr;
    int out_pieces = 0;            // K4 launches of the last chunked product
    size_t out_tiles_per = 0;      // carry tiles per K4 launch
    int spin_limit = 1 << 22;
    bool inject_wait_fault = false;
    CUtensorMap tmap_res;          // residues of A as [prime][row][column] (tma_cols)
};

// Tensor map of a context's A residues for the TMA form of the inverse column
// pass: dims (columns, rows, primes), boxes of CB columns x min(R, 256) rows.
// cuTensorMapEncodeTiled comes from the driver through the runtime's entry
// point query, so the library needs no link to libcuda.
static int encode_residue_map(bw_ctx* c) {
    using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static EncodeFn encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<EncodeFn>(fn);
    });
    if (!encode) return bw_fail(BW_ECUDA, "cuTensorMapEncodeTiled is not available");
    const bw_plan* pl = c->plan;
    const int w = pl->path == BW_PATH_P64 ? 8 : 4;
    const cuuint64_t C = (cuuint64_t)1 << pl->log_c, R = (cuuint64_t)1 << pl->log_r;
    const cuuint64_t dims[3] = {C, R, (cuuint64_t)pl->K};
    const cuuint64_t strides[2] = {C * w, C * R * w};
    const cuuint32_t box[3] = {1u << pl->log_cb, (cuuint32_t)std::min<cuuint64_t>(R, 256), 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (((cuuint64_t)box[0] * w) % 16 != 0)
        return bw_fail(BW_EINVAL, "column tile of %u x %d bytes is not a 16-byte multiple", box[0], w);
    const CUresult r = encode(&c->tmap_res,
                              w == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
                              3, c->d_res_a, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return bw_fail(BW_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return BW_OK;
}

extern "C" int bw_ctx_create(bw_ctx** out, const bw_plan* pl, void* stream) {
    bw_clear_error();
    if (!out || !pl) return bw_fail(BW_EINVAL, "NULL argument");
    *out = nullptr;
    bw_ctx* c = new bw_ctx();
    c->plan = pl;
    auto fail = [&](int rc) {
        bw_ctx_destroy(c);
        return rc;
    };
    const size_t n = (size_t)1 << pl->log_n;
    const int w = pl->path == BW_PATH_P64 ? 8 : 4;
    const size_t res_bytes = (size_t)pl->K * n * w;
    cudaError_t e;
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(bw_fail(BW_ECUDA, "stream: %s", cudaGetErrorString(e)));
        c->own_stream = true;
    }
    if ((e = cudaMalloc(&c->d_res_a, res_bytes)) != cudaSuccess ||
        (e = cudaMalloc(&c->d_res_b, res_bytes)) != cudaSuccess ||
        (e = cudaMalloc(&c->d_in, ((pl->la + pl->lb + 3) & ~(size_t)3) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&c->d_out, ((pl->la + pl->lb + 3) & ~(size_t)3) * 4)) != cudaSuccess)
        return fail(bw_fail(BW_ENOMEM, "context allocation (%zu bytes of residues x2): %s",
                            res_bytes, cudaGetErrorString(e)));
    // carry tiles cover the coefficients' words and the product's words
    // (la + lb can exceed the coefficients' words when la + lb - 1 is a
    // power of two)
    const size_t words = std::max(coef_words(pl), pl->la + pl->lb);
    c->ntiles = (words + kCarryTileWords - 1) / kCarryTileWords;
    c->state_bytes = 32 + c->ntiles * 16 + c->ntiles * 4;
    if ((e = cudaMalloc(&c->d_state, c->state_bytes)) != cudaSuccess)
        return fail(bw_fail(BW_ENOMEM, "carry state: %s", cudaGetErrorString(e)));
    if ((e = cudaMemset(c->d_state, 0, c->state_bytes)) != cudaSuccess)
        return fail(bw_fail(BW_ECUDA, "memset: %s", cudaGetErrorString(e)));
    c->cst = reinterpret_cast<CarryState*>(c->d_state);
    c->err = reinterpret_cast<uint32_t*>(c->d_state + 16);
    c->rec_x = reinterpret_cast<uint4*>(c->d_state + 32);
    c->rec_s = reinterpret_cast<uint32_t*>(c->d_state + 32 + c->ntiles * 16);
    if ((e = cudaMallocHost(&c->h_err, 16)) != cudaSuccess)
        return fail(bw_fail(BW_ENOMEM, "pinned: %s", cudaGetErrorString(e)));
    for (auto& ev : c->ev)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess)
            return fail(bw_fail(BW_ECUDA, "event: %s", cudaGetErrorString(e)));
    for (auto& ev : c->stage_ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess)
            return fail(bw_fail(BW_ECUDA, "event: %s", cudaGetErrorString(e)));
    if (pl->tma_cols) {
        const int rc = encode_residue_map(c);
        if (rc) return fail(rc);
    }
    if (pl->order) {
        std::lock_guard<std::mutex> lk(pl->order->mu);
        pl->order->contexts++;
        c->counted = true;
    }
    *out = c;
    return BW_OK;
}

extern "C" int bw_ctx_destroy(bw_ctx* c) {
    if (!c) return BW_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->counted) {
        bw_stage_order* so = c->plan->order;
        std::lock_guard<std::mutex> lk(so->mu);
        so->contexts--;
        for (int i = 0; i < 3; ++i)
            if (so->owner[i] == c) {
                so->owner[i] = nullptr;
                so->last[i] = nullptr;
            }
    }
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    for (auto& ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : c->stage_ev)
        if (ev) cudaEventDestroy(ev);
    if (c->in_stream) cudaStreamSynchronize(c->in_stream);
    if (c->out_stream) cudaStreamSynchronize(c->out_stream);
    for (auto& ev : c->in_ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : c->out_ev)
        if (ev) cudaEventDestroy(ev);
    if (c->ready_ev) cudaEventDestroy(c->ready_ev);
    if (c->out_done_ev) cudaEventDestroy(c->out_done_ev);
    if (c->in_stream) cudaStreamDestroy(c->in_stream);
    if (c->out_stream) cudaStreamDestroy(c->out_stream);
    if (c->h_err) cudaFreeHost(c->h_err);
    cudaFree(c->d_state);
    cudaFree(c->d_out);
    cudaFree(c->d_in);
    cudaFree(c->d_res_b);
    cudaFree(c->d_res_a);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return BW_OK;
}

extern "C" void* bw_ctx_stream(const bw_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" int bw_ctx_set_copy_chunks(bw_ctx* c, int chunks) {
    bw_clear_error();
    if (!c) return bw_fail(BW_EINVAL, "NULL ctx");
    if (chunks < 0 || chunks > kMaxCopyChunks)
        return bw_fail(BW_EINVAL, "copy chunks %d outside 0..%d", chunks, kMaxCopyChunks);
    c->copy_chunks = chunks;
    return BW_OK;
}

static int read_device_errors(bw_ctx* c) {
    BW_CUDA(cudaMemcpyAsync(c->h_err, c->err, 4, cudaMemcpyDeviceToHost, c->stream));
    BW_CUDA(cudaStreamSynchronize(c->stream));
    const uint32_t e = *c->h_err;
    if (e) {
        BW_CUDA(cudaMemsetAsync(c->err, 0, 4, c->stream));
        BW_CUDA(cudaStreamSynchronize(c->stream));
        if (e & 1u)
            return bw_fail(BW_ETIMEOUT, "carry look-back wait exceeded its bound (err=0x%x)", e);
        return bw_fail(BW_ECHECK, "redundant-prime reconstruction check failed (err=0x%x)", e);
    }
    return BW_OK;
}

extern "C" int bw_ctx_set_wait_limit(bw_ctx* c, int polls) {
    bw_clear_error();
    if (!c || polls < 0) return bw_fail(BW_EINVAL, "bad argument");
    c->spin_limit = polls;
    return BW_OK;
}

extern "C" int bw_ctx_inject_wait_fault(bw_ctx* c, int enable) {
    bw_clear_error();
    if (!c) return bw_fail(BW_EINVAL, "NULL ctx");
    c->inject_wait_fault = enable != 0;
    return BW_OK;
}

extern "C" int bw_ctx_sync(bw_ctx* c) {
    bw_clear_error();
    if (!c) return bw_fail(BW_EINVAL, "NULL ctx");
    BW_CUDA(cudaStreamSynchronize(c->stream));
    return read_device_errors(c);
}

// ------------------------------------------------------------------ launch

namespace {

template <class Ar>
const PlanDev<Ar>& plan_dev(const bw_plan* pl);
template <>
const PlanDev<Ar32>& plan_dev<Ar32>(const bw_plan* pl) {
    return pl->pd32;
}
template <>
const PlanDev<Ar64>& plan_dev<Ar64>(const bw_plan* pl) {
    return pl->pd64;
}

constexpr int kMaxDynSmem = 200 * 1024;

template <class Ar, bool SPLIT16>
int set_smem_attrs() {
    static std::once_flag once;
    static cudaError_t st = cudaSuccess;
    std::call_once(once, [] {
        auto set = [](const void* f) {
            cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 kMaxDynSmem);
            if (e != cudaSuccess) st = e;
        };
        set((const void*)k_fwd_col<Ar, SPLIT16, 4, true>);
        set((const void*)k_fwd_col<Ar, SPLIT16, 4, false>);
        set((const void*)k_inv_col<Ar, 4, true>);
        set((const void*)k_inv_col<Ar, 4, false>);
        set((const void*)k_row<Ar, 64, 4>);
        set((const void*)k_row<Ar, 128, 4>);
        set((const void*)k_row<Ar, 256, 4>);
        set((const void*)k_row<Ar, 512, 4>);
        set((const void*)k_row<Ar, 64, 3>);
        set((const void*)k_row<Ar, 128, 3>);
        set((const void*)k_row<Ar, 256, 3>);
        set((const void*)k_row<Ar, 512, 3>);
        if constexpr (sizeof(typename Ar::T) == 4) set((const void*)k_row<Ar, 256, 4, true>);
        if constexpr (sizeof(typename Ar::T) == 4 && !SPLIT16) {
            // 64-bit coefficients on the 32-bit path
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, true, true, false>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, false, true, false>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, true, true, true>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, false, true, true>);
        }
        set((const void*)k_mid_col<Ar, false>);
        set((const void*)k_mid_col<Ar, true>);
        set((const void*)k_inv_col_tma<Ar, 4>);
        if constexpr (sizeof(typename Ar::T) == 8) {
            set((const void*)k_fwd_col<Ar, SPLIT16, 3, true, false, true>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 3, false, false, true>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 3, true, true, true>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 3, false, true, true>);
            set((const void*)k_inv_col<Ar, 3, true>);
            set((const void*)k_inv_col<Ar, 3, false>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, true, false, true>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, false, false, true>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, true, true, true>);
            set((const void*)k_fwd_col<Ar, SPLIT16, 4, false, true, true>);
        }
    });
    if (st != cudaSuccess) return bw_fail(BW_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(st));
    return BW_OK;
}

}  // namespace

int bw_set_kernel_attrs() {
    int rc = set_smem_attrs<Ar64, false>();
    if (!rc) rc = set_smem_attrs<Ar32, true>();
    return rc;
}

namespace {

template <class Ar, int RLOG>
void launch_row(const bw_plan* pl, const PlanDev<Ar>& pd, typename Ar::T* ra,
                const typename Ar::T* rb, int sq, size_t smem, cudaStream_t s) {
    dim3 g(1u << (pl->log_r + pl->log_r2), pl->K);
    // one thread per sub-problem of a round, 64..512 threads (radix-8 rounds,
    // and radix-16 rounds on the 32-bit path: at most 256, each thread taking
    // several sub-problems, so that the CTA's registers leave room for more
    // than one CTA per SM; 2^13-point rows on the 32-bit path ran one 512-thread
    // CTA per SM at 70 registers)
    const int cap = (RLOG == 3 || sizeof(typename Ar::T) == 4) ? 256 : 512;
    const int want = std::min(cap, std::max(64, 1 << (pl->log_c - RLOG)));
    if constexpr (sizeof(typename Ar::T) == 4 && RLOG == 4) {
        if (pl->shfl_rows && want == 256) {
            k_row<Ar, 256, 4, true><<<g, 256, smem, s>>>(pd, ra, rb, sq);
            return;
        }
    }
    switch (want) {
        case 512: k_row<Ar, 512, RLOG><<<g, 512, smem, s>>>(pd, ra, rb, sq); break;
        case 256: k_row<Ar, 256, RLOG><<<g, 256, smem, s>>>(pd, ra, rb, sq); break;
        case 128: k_row<Ar, 128, RLOG><<<g, 128, smem, s>>>(pd, ra, rb, sq); break;
        default: k_row<Ar, 64, RLOG><<<g, 64, smem, s>>>(pd, ra, rb, sq); break;
    }
}

// Stage order of one host-pointer product (bw_stage_order): begin(i, s)
// makes stream s wait for stage i of the plan's previous product; end(i, s)
// records this product's stage i on s.  Off with one live context.  A
// previous product of the same context needs no wait: every stream of a
// product starts behind the context stream, which ends behind all of the
// previous product's work.
struct StageOrder {
    bw_stage_order* so = nullptr;
    const bw_ctx* c = nullptr;
    bool on = false;
    cudaError_t begin(int i, cudaStream_t s) const {
        if (!on || !so->last[i] || so->owner[i] == c) return cudaSuccess;
        return cudaStreamWaitEvent(s, so->last[i], 0);
    }
    cudaError_t end(int i, cudaStream_t s) const {
        if (!on) return cudaSuccess;
        const cudaError_t e = cudaEventRecord(c->stage_ev[i], s);
        so->last[i] = c->stage_ev[i];
        so->owner[i] = c;
        return e;
    }
};

// Host operands of a product whose copy-in is split into `chunks` column
// blocks: block k holds the words of forward-column tiles
// [k T/chunks, (k+1) T/chunks) of every row, and K1 runs over those tiles
// as soon as the block has landed.
struct HostIO {
    const uint32_t* ha = nullptr;
    const uint32_t* hb = nullptr;  // nullptr when squaring
    int chunks = 1;
    const StageOrder* order = nullptr;
};

// Copy words [w0, w1) of every row (row length wc words) of an operand of lx
// words: one 2D copy over the full rows, one plain copy of the partial last
// row's part.  Nothing at or beyond lx is read or written.
cudaError_t copy_cols(cudaStream_t s, uint32_t* dst, const uint32_t* src, size_t lx, size_t wc,
                      size_t w0, size_t w1) {
    const size_t full = lx / wc;
    cudaError_t e = cudaSuccess;
    if (full)
        e = cudaMemcpy2DAsync(dst + w0, wc * 4, src + w0, wc * 4, (w1 - w0) * 4, full,
                              cudaMemcpyHostToDevice, s);
    const size_t lo = full * wc + w0, hi = std::min(lx, full * wc + w1);
    if (e == cudaSuccess && hi > lo)
        e = cudaMemcpyAsync(dst + lo, src + lo, (hi - lo) * 4, cudaMemcpyHostToDevice, s);
    return e;
}

int ensure_copy_streams(bw_ctx* c) {
    if (c->in_stream) return BW_OK;
    BW_CUDA(cudaStreamCreateWithFlags(&c->in_stream, cudaStreamNonBlocking));
    BW_CUDA(cudaStreamCreateWithFlags(&c->out_stream, cudaStreamNonBlocking));
    for (auto& ev : c->in_ev) BW_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (auto& ev : c->out_ev) BW_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    BW_CUDA(cudaEventCreateWithFlags(&c->ready_ev, cudaEventDisableTiming));
    BW_CUDA(cudaEventCreateWithFlags(&c->out_done_ev, cudaEventDisableTiming));
    return BW_OK;
}

// Chunks of a host product's copies: the context's setting, else automatic:
// whole copies while the plan's stage order is on (the products in flight
// already hide each other's copies, and K1 and K4 in pieces cost 3-11% of
// that pipeline's throughput), otherwise 8 from 2^23 product words and 4
// from 2^21 (measured best; below 2^21 words the copies take less time than
// the extra launches cost).  Capped by the forward-column tiles per operand
// and rounded down to a power of two so that it divides them.  1 means whole
// copies on the context stream.
int copy_chunks_for(const bw_ctx* c, bool ordered) {
    const bw_plan* pl = c->plan;
    const size_t M = pl->la + pl->lb;
    int want = c->copy_chunks;
    if (want == 0)
        want = ordered ? 1 : M >= ((size_t)1 << 23) ? 8 : M >= ((size_t)1 << 21) ? 4 : 1;
    const int tiles1 = 1 << (pl->log_c + pl->log_r2 - pl->log_cb1);
    want = std::min(std::min(want, tiles1), kMaxCopyChunks);
    int S = 1;
    while (S * 2 <= want) S *= 2;
    const int cpw = (pl->path == BW_PATH_P32 && !pl->w64) ? 2 : 1;
    if (S > 1 && ((tiles1 / S) << pl->log_cb1) % cpw) S = 1;
    return S;
}

// Enqueue K1..K3 (the transform part) for one product.  With io (chunks > 1)
// the operands' copy-in runs on the context's copy stream in column blocks
// and K1 runs block by block behind it.
template <class Ar, bool SPLIT16, bool W64 = false>
int enqueue_transform(bw_ctx* c, const uint32_t* a, const uint32_t* b, bool square,
                      bool timing, const HostIO* io = nullptr) {
    using T = typename Ar::T;
    const bw_plan* pl = c->plan;
    const PlanDev<Ar>& pd = plan_dev<Ar>(pl);
    int rc = set_smem_attrs<Ar, SPLIT16>();
    if (rc) return rc;
    const int R = 1 << pl->log_r, C = 1 << pl->log_c, CB = 1 << pl->log_cb;
    T* ra = reinterpret_cast<T*>(c->d_res_a);
    T* rb = reinterpret_cast<T*>(c->d_res_b);
    const bool ts = pl->tw_smem_r != 0;
    const size_t tw_bytes = ts ? (size_t)R * sizeof(Tw<T>) : 0;

    const int CB1 = 1 << pl->log_cb1;
    // the 64-bit path stages the coefficients inside the residue tile and
    // runs one prime per CTA (grid.x = tile * K + prime); so does the 32-bit
    // path with 64-bit coefficients when asked (BW_PLAN_K1_ONE_PRIME); the
    // 32-bit path keeps a u16 (16-bit) or u64 (64-bit coefficients) copy
    constexpr bool PP = sizeof(T) == 8;
    const bool pp32 = W64 && sizeof(T) == 4 && pl->k1_pp;
    // (64-bit coefficients on the 32-bit path: the u64 copy holds the loaded
    // rows only, half the tile when both operands fill at most half of it)
    const size_t coef_rows = (W64 && sizeof(T) == 4 && pl->coef_half) ? (size_t)R / 2 : R;
    const size_t smem1 = tw_bytes + tile_elems((size_t)R * CB1) * sizeof(T) +
                         coef_rows * CB1 * ((PP || pp32) ? 0 : SPLIT16 ? 2 : W64 ? 8 : 4) +
                         (W64 && sizeof(T) == 4 && !pp32 ? 16 : 0);
    // K1 takes coefficient counts, or word counts for 64-bit coefficients
    const size_t in_a = W64 ? pl->la : pl->nca, in_b = W64 ? pl->lb : pl->ncb;
    const int cols_outer = 1 << (pl->log_c + pl->log_r2);
    const int tiles1 = cols_outer / CB1;
    const unsigned zt = (pl->zt_a ? 1u : 0u) | (pl->zt_b ? 2u : 0u);
    auto k1 = [&](int tile0, int ntiles) {
        dim3 g1(ntiles * ((PP || pp32) ? pl->K : 1), 1, square ? 1 : 2);
        if constexpr (W64 && sizeof(T) == 4) {
            if (pp32) {
                if (ts) {
                    k_fwd_col<Ar, SPLIT16, 4, true, true, true>
                        <<<g1, kColThreads, smem1, c->stream>>>(pd, a, in_a, b, in_b, ra, rb, zt,
                                                                tile0);
                } else {
                    k_fwd_col<Ar, SPLIT16, 4, false, true, true>
                        <<<g1, kColThreads, smem1, c->stream>>>(pd, a, in_a, b, in_b, ra, rb, zt,
                                                                tile0);
                }
                return;
            }
        }
        if constexpr (PP) {
            if (pl->rlog_col == 3) {
                if (ts) {
                    k_fwd_col<Ar, SPLIT16, 3, true, W64, PP><<<g1, kColThreads, smem1, c->stream>>>(
                        pd, a, in_a, b, in_b, ra, rb, zt, tile0);
                } else {
                    k_fwd_col<Ar, SPLIT16, 3, false, W64, PP>
                        <<<g1, kColThreads, smem1, c->stream>>>(pd, a, in_a, b, in_b, ra, rb, zt,
                                                                tile0);
                }
                return;
            }
        }
        if (ts) {
            k_fwd_col<Ar, SPLIT16, 4, true, W64, PP><<<g1, kColThreads, smem1, c->stream>>>(
                pd, a, in_a, b, in_b, ra, rb, zt, tile0);
        } else {
            k_fwd_col<Ar, SPLIT16, 4, false, W64, PP><<<g1, kColThreads, smem1, c->stream>>>(
                pd, a, in_a, b, in_b, ra, rb, zt, tile0);
        }
    };
    if (!io || io->chunks <= 1) {
        k1(0, tiles1);
    } else {
        // the copy stream starts where the context stream is (the previous
        // product has read the staging buffer); block k: copy, event, K1
        // words per row of coefficients: cols / 2 (16-bit), cols (32-bit),
        // 2 cols (64-bit coefficients)
        const int S = io->chunks, per = tiles1 / S, cpw = SPLIT16 ? 2 : 1;
        const size_t wpc = W64 ? 2 : 1;
        const size_t wc = (size_t)cols_outer * wpc / cpw;
        uint32_t* da = const_cast<uint32_t*>(a);
        uint32_t* db = const_cast<uint32_t*>(b);
        BW_CUDA(cudaEventRecord(c->ready_ev, c->stream));
        BW_CUDA(cudaStreamWaitEvent(c->in_stream, c->ready_ev, 0));
        BW_CUDA(io->order->begin(0, c->in_stream));
        BW_CUDA(io->order->begin(1, c->stream));
        for (int k = 0; k < S; ++k) {
            const size_t w0 = ((size_t)k * per << pl->log_cb1) * wpc / cpw;
            const size_t w1 = ((size_t)(k + 1) * per << pl->log_cb1) * wpc / cpw;
            BW_CUDA(copy_cols(c->in_stream, da, io->ha, pl->la, wc, w0, w1));
            if (!square) BW_CUDA(copy_cols(c->in_stream, db, io->hb, pl->lb, wc, w0, w1));
            BW_CUDA(cudaEventRecord(c->in_ev[k], c->in_stream));
            if (k == S - 1) BW_CUDA(io->order->end(0, c->in_stream));
            BW_CUDA(cudaStreamWaitEvent(c->stream, c->in_ev[k], 0));
            k1(k * per, per);
        }
    }
    // three passes: middle column pass with the outer twiddle
    const int CB2 = 1 << pl->log_cb2;
    const size_t smem_mid = (((size_t)1 << pl->log_r2) + CB2) * sizeof(Tw<T>) +
                            tile_elems((size_t)CB2 << pl->log_r2) * sizeof(T);
    if (pl->log_r2) {
        dim3 gm(C / CB2, R, pl->K * (square ? 1 : 2));
        k_mid_col<Ar, false><<<gm, kColThreads, smem_mid, c->stream>>>(pd, ra, rb);
    }
    if (timing) cudaEventRecord(c->ev[2], c->stream);

    const int la = pl->log_c / 2;
    const size_t ntab = 2 * (((size_t)1 << la) + ((size_t)C >> la));
    const size_t smem2 = ntab * sizeof(Tw<T>) + tile_elems(C) * sizeof(T) * (square ? 1 : 2);
    const T* rbs = square ? ra : rb;
    const int sq = square ? 1 : 0;
    if (pl->rlog_row == 3) {
        launch_row<Ar, 3>(pl, pd, ra, rbs, sq, smem2, c->stream);
    } else {
        launch_row<Ar, 4>(pl, pd, ra, rbs, sq, smem2, c->stream);
    }
    if (timing) cudaEventRecord(c->ev[3], c->stream);

    if (pl->log_r2) {
        dim3 gm(C / CB2, R, pl->K);
        k_mid_col<Ar, true><<<gm, kColThreads, smem_mid, c->stream>>>(pd, ra, ra);
    }
    const size_t smem3 = tw_bytes + tile_elems((size_t)R * CB) * sizeof(T);
    dim3 g3(cols_outer / CB, pl->K);
    bool inv_done = false;
    if (pl->tma_cols) {
        k_inv_col_tma<Ar, 4><<<g3, kColThreads, (size_t)R * CB * sizeof(T) + 128, c->stream>>>(
            pd, ra, c->cst, c->tmap_res, c->err, c->spin_limit);
        inv_done = true;
    }
    if constexpr (PP) {
        if (!inv_done && pl->rlog_col == 3) {
            if (ts) {
                k_inv_col<Ar, 3, true><<<g3, kColThreads, smem3, c->stream>>>(pd, ra, c->cst);
            } else {
                k_inv_col<Ar, 3, false><<<g3, kColThreads, smem3, c->stream>>>(pd, ra, c->cst);
            }
            inv_done = true;
        }
    }
    if (!inv_done) {
        if (ts) {
            k_inv_col<Ar, 4, true><<<g3, kColThreads, smem3, c->stream>>>(pd, ra, c->cst);
        } else {
            k_inv_col<Ar, 4, false><<<g3, kColThreads, smem3, c->stream>>>(pd, ra, c->cst);
        }
    }
    if (timing) cudaEventRecord(c->ev[4], c->stream);
    BW_CUDA(cudaGetLastError());
    return BW_OK;
}

template <class Ar, bool SPLIT16, bool W64 = false>
int enqueue_carry(bw_ctx* c, uint32_t* out, int pieces = 1) {
    using T = typename Ar::T;
    const bw_plan* pl = c->plan;
    const PlanDev<Ar>& pd = plan_dev<Ar>(pl);
    const size_t n = (size_t)1 << pl->log_n;
    const size_t NL = W64 ? 2 * n : n / (SPLIT16 ? 2 : 1);
    const size_t M = pl->la + pl->lb;
    uint32_t epoch = 1;
    if (!c->capturing) {
        if (++c->epoch >= (1u << 28)) {
            c->epoch = 2;
            BW_CUDA(cudaMemsetAsync(c->d_state + 32, 0, c->state_bytes - 32, c->stream));
        }
        epoch = c->epoch;
    }
    if (c->ntiles > 1) {
        const unsigned nb = (unsigned)((c->ntiles - 1 + 255) / 256);
        k_carry_bounds<Ar, SPLIT16, W64><<<nb, 256, 0, c->stream>>>(
            pd, reinterpret_cast<const T*>(c->d_res_a), NL, c->rec_x, (uint32_t)c->ntiles,
            epoch);
    }
    // Tiles come from a ticket counter in launch order, so `pieces` launches
    // in a row cover tiles [k per, (k+1) per) each; out_ev[k] marks the end of
    // launch k, after which its words are final and can be copied out.
    const size_t per = (c->ntiles + pieces - 1) / pieces;
    c->out_pieces = 0;
    c->out_tiles_per = per;
    if (pieces == 1 && !c->inject_wait_fault) {
        // one piece: the words pass (no waits between tiles) and the carry
        // fix; the look-back form below stays for pieces that are copied out
        // one by one and for the fault-injection hook, whose waits it tests
        k_garner_words<Ar, SPLIT16, W64><<<(unsigned)c->ntiles, kCarryThreads, 0, c->stream>>>(
            pd, reinterpret_cast<const T*>(c->d_res_a), out, M, NL, c->rec_x, c->rec_s, c->err);
        if (c->ntiles > 1)
            k_carry_fix<<<1, kFixThreads, 0, c->stream>>>(c->rec_s, (uint32_t)c->ntiles, out, M);
        c->out_pieces = 1;
        BW_CUDA(cudaGetLastError());
        return BW_OK;
    }
    for (size_t t0 = 0; t0 < c->ntiles; t0 += per) {
        const unsigned nb = (unsigned)std::min(per, c->ntiles - t0);
        k_garner_carry<Ar, SPLIT16, W64><<<nb, kCarryThreads, 0, c->stream>>>(
            pd, reinterpret_cast<const T*>(c->d_res_a), out, M, NL, c->cst, c->rec_x, c->rec_s,
            epoch, c->inject_wait_fault ? epoch + (1u << 27) : epoch, c->err,
            c->spin_limit);
        if (pieces > 1) BW_CUDA(cudaEventRecord(c->out_ev[c->out_pieces], c->stream));
        c->out_pieces++;
    }
    BW_CUDA(cudaGetLastError());
    return BW_OK;
}

int enqueue_product(bw_ctx* c, const uint32_t* a, const uint32_t* b, uint32_t* out,
                    bool square, bool timing, const HostIO* io = nullptr) {
    const bw_plan* pl = c->plan;
    const int pieces = io ? io->chunks : 1;
    int rc;
    if (pl->w64 && pl->path == BW_PATH_P32) {
        rc = enqueue_transform<Ar32, false, true>(c, a, b, square, timing, io);
        if (!rc) rc = enqueue_carry<Ar32, false, true>(c, out, pieces);
    } else if (pl->w64) {
        rc = enqueue_transform<Ar64, false, true>(c, a, b, square, timing, io);
        if (!rc) rc = enqueue_carry<Ar64, false, true>(c, out, pieces);
    } else if (pl->path == BW_PATH_P64) {
        rc = enqueue_transform<Ar64, false>(c, a, b, square, timing, io);
        if (!rc) rc = enqueue_carry<Ar64, false>(c, out, pieces);
    } else {
        rc = enqueue_transform<Ar32, true>(c, a, b, square, timing, io);
        if (!rc) rc = enqueue_carry<Ar32, true>(c, out, pieces);
    }
    return rc;
}

float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace

// Device-pointer product through a CUDA graph of the whole pipeline (look-back
// records cleared, K1..K4), captured on first use and replayed while a, b,
// out and the squaring choice stay the same.  Returns 1 when a graph cannot
// be used (the stream is already being captured by the caller).
static int launch_graph(bw_ctx* c, const uint32_t* a, const uint32_t* b, uint32_t* out, bool sq) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone)
        return 1;
    if (!c->gexec || c->g_a != a || c->g_b != b || c->g_out != out || c->g_sq != sq) {
        if (c->gexec) {
            cudaGraphExecDestroy(c->gexec);
            c->gexec = nullptr;
        }
        int rc = bw_set_kernel_attrs();
        if (rc) return rc;
        BW_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->capturing = true;
        cudaError_t e = cudaMemsetAsync(c->d_state + 32, 0, c->state_bytes - 32, c->stream);
        rc = e == cudaSuccess ? enqueue_product(c, a, b, out, sq, false) : BW_OK;
        c->capturing = false;
        cudaGraph_t g = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
        if (rc || e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (rc) return rc;
            return bw_fail(BW_ECUDA, "graph capture: %s",
                           cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        e = cudaGraphInstantiate(&c->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            c->gexec = nullptr;
            return bw_fail(BW_ECUDA, "graph instantiate: %s", cudaGetErrorString(e));
        }
        c->g_a = a;
        c->g_b = b;
        c->g_out = out;
        c->g_sq = sq;
    }
    BW_CUDA(cudaGraphLaunch(c->gexec, c->stream));
    return BW_OK;
}

static int do_multiply(bw_ctx* c, const uint32_t* a, size_t la, const uint32_t* b, size_t lb,
                       uint32_t* out, size_t lc, unsigned flags, bw_timing* tm, bool square) {
    bw_clear_error();
    if (!c || !a || !out) return bw_fail(BW_EINVAL, "NULL argument");
    const bw_plan* pl = c->plan;
    if (square) {
        b = a;
        lb = la;
    }
    if (!b) return bw_fail(BW_EINVAL, "NULL b");
    if (la != pl->la || lb != pl->lb)
        return bw_fail(BW_EINVAL, "operand sizes %zu x %zu do not match the plan (%zu x %zu)", la,
                       lb, pl->la, pl->lb);
    const size_t M = la + lb;
    if (lc < M) return bw_fail(BW_EINVAL, "output has %zu words, needs %zu", lc, M);
    const bool sq = square || (a == b && la == lb);
    const bool timing = tm != nullptr;
    if ((flags & BW_PTR_HOST_ASYNC) && ((flags & BW_PTR_DEVICE) || timing))
        return bw_fail(BW_EINVAL, "BW_PTR_HOST_ASYNC takes host pointers and no timing");
    if (timing) cudaEventRecord(c->ev[0], c->stream);
    int rc;
    if (flags & BW_PTR_DEVICE) {
        if (!timing && !c->inject_wait_fault) {
            rc = launch_graph(c, a, b, out, sq);
            if (rc <= 0) return rc;  // 1: fall back to direct launches
        }
        if (timing) cudaEventRecord(c->ev[1], c->stream);
        rc = enqueue_product(c, a, b, out, sq, timing);
        if (rc) return rc;
        if (timing) {
            cudaEventRecord(c->ev[5], c->stream);
            cudaEventRecord(c->ev[6], c->stream);
            BW_CUDA(cudaEventSynchronize(c->ev[6]));
        }
    } else {
        // With several live contexts on the plan, each stage waits for the
        // same stage of the plan's previous product (bw_stage_order).  The
        // lock also keeps the three stages of one call together in that order.
        bw_stage_order* so = pl->order;
        std::unique_lock<std::mutex> lk;
        if (so) lk = std::unique_lock<std::mutex>(so->mu);
        StageOrder order;
        order.so = so;
        order.c = c;
        order.on = so && so->contexts > 1;
        const uint32_t* db = sq ? c->d_in : c->d_in + la;
        // large products without stage times: copies in chunks that overlap
        // K1 (copy-in by column blocks) and K4 (copy-out by word ranges)
        const int chunks = timing ? 1 : copy_chunks_for(c, order.on);
        if (chunks > 1) {
            rc = ensure_copy_streams(c);
            if (rc) return rc;
            HostIO io;
            io.ha = a;
            io.hb = sq ? nullptr : b;
            io.chunks = chunks;
            io.order = &order;
            rc = enqueue_product(c, c->d_in, db, c->d_out, sq, false, &io);
            if (rc) return rc;
            BW_CUDA(order.end(1, c->stream));
            BW_CUDA(order.begin(2, c->out_stream));
            const size_t step = c->out_tiles_per * kCarryTileWords;
            for (int k = 0; k < c->out_pieces; ++k) {
                BW_CUDA(cudaStreamWaitEvent(c->out_stream, c->out_ev[k], 0));
                const size_t lo = (size_t)k * step, hi = std::min(M, lo + step);
                if (hi > lo)
                    BW_CUDA(cudaMemcpyAsync(out + lo, c->d_out + lo, (hi - lo) * 4,
                                            cudaMemcpyDeviceToHost, c->out_stream));
            }
            BW_CUDA(order.end(2, c->out_stream));
            BW_CUDA(cudaEventRecord(c->out_done_ev, c->out_stream));
            BW_CUDA(cudaStreamWaitEvent(c->stream, c->out_done_ev, 0));
        } else {
            BW_CUDA(order.begin(0, c->stream));
            BW_CUDA(cudaMemcpyAsync(c->d_in, a, la * 4, cudaMemcpyHostToDevice, c->stream));
            if (!sq)
                BW_CUDA(cudaMemcpyAsync(c->d_in + la, b, lb * 4, cudaMemcpyHostToDevice,
                                        c->stream));
            BW_CUDA(order.end(0, c->stream));
            BW_CUDA(order.begin(1, c->stream));
            if (timing) cudaEventRecord(c->ev[1], c->stream);
            rc = enqueue_product(c, c->d_in, db, c->d_out, sq, timing);
            if (rc) return rc;
            if (timing) cudaEventRecord(c->ev[5], c->stream);
            BW_CUDA(order.end(1, c->stream));
            BW_CUDA(order.begin(2, c->stream));
            BW_CUDA(cudaMemcpyAsync(out, c->d_out, M * 4, cudaMemcpyDeviceToHost, c->stream));
            BW_CUDA(order.end(2, c->stream));
            if (timing) cudaEventRecord(c->ev[6], c->stream);
        }
        if (lk.owns_lock()) lk.unlock();
        if (flags & BW_PTR_HOST_ASYNC) return BW_OK;  // bw_ctx_sync reports errors
        rc = read_device_errors(c);
        if (rc) return rc;
    }
    if (timing) {
        tm->h2d_ms = ev_ms(c->ev[0], c->ev[1]);
        tm->fwd_ms = ev_ms(c->ev[1], c->ev[2]);
        tm->mul_ms = ev_ms(c->ev[2], c->ev[3]);
        tm->intt_ms = ev_ms(c->ev[3], c->ev[4]);
        tm->crt_carry_ms = ev_ms(c->ev[4], c->ev[5]);
        tm->d2h_ms = ev_ms(c->ev[5], c->ev[6]);
        tm->total_ms = ev_ms(c->ev[0], c->ev[6]);
    }
    return BW_OK;
}

extern "C" int bw_multiply(bw_ctx* c, const uint32_t* a, size_t la, const uint32_t* b, size_t lb,
                           uint32_t* out, size_t lc, unsigned flags, bw_timing* tm) {
    return do_multiply(c, a, la, b, lb, out, lc, flags, tm, false);
}

extern "C" int bw_square(bw_ctx* c, const uint32_t* a, size_t la, uint32_t* out, size_t lc,
                         unsigned flags, bw_timing* tm) {
    return do_multiply(c, a, la, nullptr, la, out, lc, flags, tm, true);
}

// ------------------------------------------------------------------ Garner dump

namespace {
template <class Ar, bool SPLIT16>
__global__ void k_garner_dump(const PlanDev<Ar> P, const typename Ar::T* __restrict__ res,
                              uint32_t* __restrict__ words, size_t n) {
    using T = typename Ar::T;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Ar a1 = P.pr[1].ar;
    const GarnerDev<Ar>& G = P.gar;
    const T r0 = res[i], r1 = res[n + i];
    const T r0m1 = a1.red1(a1.shoup(r0, 1, P.pr[1].one_q));
    const T t1 = r1 >= r0m1 ? r1 - r0m1 : r1 + a1.p - r0m1;
    const T k1 = a1.red1(a1.shoup(t1, G.inv1, G.inv1q));
    const unsigned __int128 x = (unsigned __int128)G.p0 * k1 + r0;
    words[3 * i] = (uint32_t)x;
    words[3 * i + 1] = (uint32_t)(x >> 32);
    words[3 * i + 2] = (uint32_t)(x >> 64);
}
}  // namespace

extern "C" int bw_multiply_coeffs(bw_ctx* c, const uint32_t* a, size_t la, const uint32_t* b,
                                  size_t lb, uint32_t* words, size_t n_words) {
    bw_clear_error();
    if (!c || !a || !b || !words) return bw_fail(BW_EINVAL, "NULL argument");
    const bw_plan* pl = c->plan;
    if (la != pl->la || lb != pl->lb) return bw_fail(BW_EINVAL, "operand sizes do not match plan");
    if (pl->w64)
        return bw_fail(BW_EINVAL,
                       "the coefficient dump follows the reference's 32-bit coefficients: make "
                       "the plan with num_primes 2 or 3");
    const size_t n = (size_t)1 << pl->log_n;
    if (n_words < 3 * n) return bw_fail(BW_EINVAL, "words needs 3*n = %zu entries", 3 * n);
    uint32_t* d_words = nullptr;
    BW_CUDA(cudaMalloc(&d_words, 3 * n * 4));
    int rc = BW_OK;
    const bool sq = (a == b && la == lb);
    cudaMemcpyAsync(c->d_in, a, la * 4, cudaMemcpyHostToDevice, c->stream);
    if (!sq) cudaMemcpyAsync(c->d_in + la, b, lb * 4, cudaMemcpyHostToDevice, c->stream);
    const uint32_t* db = sq ? c->d_in : c->d_in + la;
    if (pl->path == BW_PATH_P64) {
        rc = enqueue_transform<Ar64, false>(c, c->d_in, db, sq, false);
        if (!rc)
            k_garner_dump<Ar64, false><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
                pl->pd64, reinterpret_cast<const uint64_t*>(c->d_res_a), d_words, n);
    } else {
        rc = enqueue_transform<Ar32, true>(c, c->d_in, db, sq, false);
        if (!rc)
            k_garner_dump<Ar32, true><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(
                pl->pd32, reinterpret_cast<const uint32_t*>(c->d_res_a), d_words, n);
    }
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(words, d_words, 3 * n * 4, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) rc = bw_fail(BW_ECUDA, "coeff dump: %s", cudaGetErrorString(e));
    }
    cudaFree(d_words);
    return rc;
}

// ------------------------------------------------------------------ misc ABI

extern "C" int bw_abi_version(void) { return BW_ABI_VERSION; }

extern "C" const char* bw_last_error(void) { return g_last_error.c_str(); }

extern "C" int bw_limits(int path, int num_primes, bw_limits_info* o) {
    bw_clear_error();
    if (!o) return bw_fail(BW_EINVAL, "NULL out");
    if (path == BW_PATH_AUTO) path = BW_PATH_P64;
    if (path != BW_PATH_P32 && path != BW_PATH_P64) return bw_fail(BW_EINVAL, "unknown path");
    const int K = num_primes == 0 ? 2 : num_primes;
    if (K < 2 || K > 3) return bw_fail(BW_EINVAL, "num_primes must be 2 or 3");
    o->path = path;
    o->num_primes = K;
    o->max_log_n = bw_path_max_log_n(path, K);
    const int cpw = path == BW_PATH_P32 ? 2 : 1;
    o->max_square_words = ((size_t)1 << (o->max_log_n - 1)) / cpw;
    return BW_OK;
}

extern "C" int bw_size_supported(int path, int num_primes, size_t la, size_t lb) {
    bw_clear_error();
    int K = 0;
    bool w64 = false;
    const int rc = resolve_plan(path, num_primes, la, lb, 0, &path, &K, &w64);
    if (rc) return rc;
    return w64 ? bw_check_size_w64(la, lb, nullptr, path)
               : bw_check_size(path, K, la, lb, nullptr);
}

// Plans and contexts of recent one-shot sizes.  The reference builds and
// uploads its tables and allocates its context on every host_multiply_merge
// call (src/host_multiply.cpp:27-86); here a repeated size reuses them.  An
// entry in use by one thread is skipped by the others (they build their own,
// which then competes for the slot).  Least recently used entries go first
// when a new one would exceed the device-memory limit.  Entries are never
// freed at process exit (the CUDA runtime may already be gone by then).
namespace {
struct OnceEntry {
    int device = 0, path = 0;
    size_t la = 0, lb = 0, bytes = 0;
    bw_plan* pl = nullptr;
    bw_ctx* cx = nullptr;
    uint64_t last_use = 0;
    bool busy = false;
};
std::mutex g_once_mu;
std::vector<OnceEntry>* g_once = new std::vector<OnceEntry>();
size_t g_once_limit = (size_t)4 << 30;
uint64_t g_once_clock = 0;

// Frees idle entries, least recently used first, until `need` more bytes fit
// under the limit.  Called with g_once_mu held.
void once_evict(size_t need) {
    for (;;) {
        size_t used = 0;
        for (const auto& e : *g_once) used += e.bytes;
        if (used + need <= g_once_limit) return;
        int victim = -1;
        for (int i = 0; i < (int)g_once->size(); ++i)
            if (!(*g_once)[i].busy &&
                (victim < 0 || (*g_once)[i].last_use < (*g_once)[victim].last_use))
                victim = i;
        if (victim < 0) return;
        bw_ctx_destroy((*g_once)[victim].cx);
        bw_plan_destroy((*g_once)[victim].pl);
        g_once->erase(g_once->begin() + victim);
    }
}
}  // namespace

extern "C" int bw_host_once_cache_limit(size_t bytes) {
    bw_clear_error();
    std::lock_guard<std::mutex> lk(g_once_mu);
    g_once_limit = bytes;
    once_evict(0);
    return BW_OK;
}

extern "C" int bw_multiply_host_once(const uint32_t* a, size_t la, const uint32_t* b, size_t lb,
                                     uint32_t* c, size_t lc, int path, float* elapsed_ms) {
    const auto t0 = std::chrono::high_resolution_clock::now();
    int device = 0;
    cudaGetDevice(&device);
    bool hit = false;  // got is a copy of a cache entry marked busy
    OnceEntry got;
    {
        std::lock_guard<std::mutex> lk(g_once_mu);
        for (auto& e : *g_once)
            if (!e.busy && e.device == device && e.path == path && e.la == la && e.lb == lb) {
                e.busy = true;
                hit = true;
                got = e;
                break;
            }
    }
    int rc = BW_OK;
    if (!hit) {
        got.device = device;
        got.path = path;
        got.la = la;
        got.lb = lb;
        rc = bw_plan_create(&got.pl, path, la, lb, 0, 0);
        if (!rc) rc = bw_ctx_create(&got.cx, got.pl, nullptr);
        if (!rc) got.bytes = ctx_bytes(got.pl) + got.pl->table_bytes;
    }
    if (!rc) rc = bw_multiply(got.cx, a, la, b, lb, c, lc, BW_PTR_HOST, nullptr);
    const std::string err = rc ? g_last_error : std::string();
    {
        std::lock_guard<std::mutex> lk(g_once_mu);
        if (hit) {
            // other calls may have moved the entries: find it by its context
            for (auto& e : *g_once)
                if (e.cx == got.cx) {
                    e.busy = false;
                    e.last_use = ++g_once_clock;
                }
        } else if (got.cx && got.bytes <= g_once_limit) {
            once_evict(got.bytes);
            size_t used = 0;
            for (const auto& e : *g_once) used += e.bytes;
            if (used + got.bytes <= g_once_limit) {
                got.last_use = ++g_once_clock;
                got.busy = false;
                g_once->push_back(got);
                got.cx = nullptr;
                got.pl = nullptr;
            }
        }
    }
    if (got.cx && !hit) bw_ctx_destroy(got.cx);
    if (got.pl && !hit) bw_plan_destroy(got.pl);
    if (rc) g_last_error = err;
    const auto t1 = std::chrono::high_resolution_clock::now();
    if (elapsed_ms) *elapsed_ms = std::chrono::duration<float, std::milli>(t1 - t0).count();
    return rc;
}
