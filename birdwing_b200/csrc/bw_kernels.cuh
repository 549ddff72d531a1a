// bw_kernels.cuh -- device side of the product pipeline (both prime paths).
//
// A product of two operands is computed as a cyclic convolution of length
// n = 2^log_n = R * C per prime with a 4-step NTT:
//
//   K1 fwd_col   per operand, per tile of CB columns of the R x C matrix:
//                limb split + virtual zero pad, R-point forward NTT down each
//                column, inter-pass twiddle w_n^(c * bitrev(r)), write.
//   K2 row       per prime, per row: C-point forward NTT of the A row and the
//                B row, pointwise Montgomery product, C-point inverse NTT,
//                inverse twiddle (scaled by n^-1 * 2^bits), write in place.
//   K3 inv_col   per prime, per column tile: R-point inverse NTT down each
//                column, full reduction, write residues in natural order.
//   K4 garner_carry  per tile of 2048 output words: Garner reconstruction of
//                every coefficient from its K residues, carry generation, and
//                carry propagation across tiles by decoupled look-back.
//
// Forward transforms are Cooley-Tukey with natural-order input and
// bit-reversed output ("CT-BR"); inverse transforms are Gentleman-Sande with
// bit-reversed input and natural output.  Stage s (m = 2^s groups) uses the
// twiddle table entries W[m .. 2m), W[m + i] = w_{2m}^{bitrev_s(i)}.  Each
// round processes up to four stages in registers (radix 16); rounds exchange
// data through swizzled shared memory.
//
// The reference runs these stages as separate kernels with separate HBM
// passes: zero_pad (src/zero_pad.cu:3-57), GPU-NTT forward/inverse
// (src/gpu_ntt.cu:577-581,742-747), pointwise_mul_kernel
// (src/gpu_ntt.cu:216-238), crt_combine_kernel (src/crt_gpu.cu:157-276) and the
// three carry kernels (src/carry_prop.cu:8-211).
#pragma once
#include <cstdint>
#include "bw_arith.cuh"

namespace bw {

constexpr int kMaxPrimes = 3;
constexpr int kCarryThreads = 256;
constexpr int kCarryWordsPerThread = 8;
constexpr int kCarryTileWords = kCarryThreads * kCarryWordsPerThread;  // 2048
constexpr int kColThreads = 256;

// Per-prime device view of a plan.
template <class Ar>
struct PrimeDev {
    using T = typename Ar::T;
    const Tw<T>* WRf;  // column (R-point) forward stage twiddles, R entries
    const Tw<T>* WRi;  // column inverse
    const Tw<T>* WCf;  // row (C-point) forward, C entries
    const Tw<T>* WCi;  // row inverse
    const Tw<T>* TLf;  // inter-pass twiddle w_n^e, e = eh*2^LO + el: low table
    const Tw<T>* THf;  //   high table
    const Tw<T>* TLi;  // inverse inter-pass twiddle, low table
    const Tw<T>* THi;  //   high table, scaled by n^-1 * 2^bits
    Ar ar;
    T one_q;           // floor(2^bits / p): Shoup companion of 1 (x mod p)
};

// Garner constants (reference: CRTGarnerParams, include/crt_gpu.h:11-17,
// computed by compute_garner_params, src/crt_gpu.cu:70-105).
template <class Ar>
struct GarnerDev {
    using T = typename Ar::T;
    T inv1, inv1q;      // p0^-1 mod p1
    T p0m2, p0m2q;      // p0 mod p2
    T inv2, inv2q;      // (p0 p1)^-1 mod p2
    uint64_t p0;        // p0 as an integer
};

template <class Ar>
struct PlanDev {
    PrimeDev<Ar> pr[kMaxPrimes];
    GarnerDev<Ar> gar;
    int K;
    int log_n, log_r, log_c, lo;  // lo: split of the inter-pass exponent
    int log_cb;                   // column tile width CB = 2^log_cb
};

// Carry look-back state of one context.
struct CarryState {
    uint32_t counter;   // dynamic tile ticket (reset by K3 before every K4)
    uint32_t pad[3];
};

// ------------------------------------------------------------------ helpers

template <typename T>
__device__ __forceinline__ int swz(int e) {
    if constexpr (sizeof(T) == 8) {
        return e ^ ((e >> 4) & 15);
    } else {
        return e ^ ((e >> 4) & 31);
    }
}

__device__ __forceinline__ uint32_t bitrev(uint32_t x, int bits) {
    return bits == 0 ? 0u : (__brev(x) >> (32 - bits));
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Round schedule of a 2^log_len-point transform: the remainder round (fewer
// than four stages) comes first, where the sub-problem stride is largest and
// shared-memory accesses are conflict-free; all later rounds are radix 16.
struct Sched {
    int n;
    int s0[8];
    int rl[8];
};
__host__ __device__ __forceinline__ Sched make_sched(int log_len) {
    Sched s;
    s.n = 0;
    int at = 0;
    const int rem = log_len & 3;
    if (rem) {
        s.s0[0] = 0;
        s.rl[0] = rem;
        s.n = 1;
        at = rem;
    }
    while (at < log_len) {
        s.s0[s.n] = at;
        s.rl[s.n] = 4;
        s.n++;
        at += 4;
    }
    return s;
}

// Forward CT stages s0 .. s0+RL-1 on one sub-problem of 2^RL elements that
// belongs to group g of stage s0.  With zt (first round of a zero-padded
// column) the elements of the second half are zero and stage 0 (twiddle 1)
// reduces to duplicating the first half.
template <class Ar, int RL>
__device__ __forceinline__ void ct_stages(typename Ar::T* x, int s0, int g,
                                          const Tw<typename Ar::T>* __restrict__ W,
                                          const Ar& ar, bool zt) {
    using T = typename Ar::T;
#pragma unroll
    for (int l = 0; l < RL; ++l) {
        const int h = 1 << (RL - l - 1);
        if (l == 0 && zt) {
#pragma unroll
            for (int u = 0; u < h; ++u) x[u + h] = x[u];
            continue;
        }
        const Tw<T>* Ws = W + (1 << (s0 + l)) + (g << l);
#pragma unroll
        for (int q = 0; q < (1 << l); ++q) {
            const Tw<T> w = ld_tw(Ws + q);
#pragma unroll
            for (int u = 0; u < h; ++u) {
                const int k = (q << (RL - l)) + u;
                ar.ct(x[k], x[k + h], w.w, w.wq);
            }
        }
    }
}

// Inverse GS stages s0+RL-1 down to s0 (the mirror of ct_stages).
template <class Ar, int RL>
__device__ __forceinline__ void gs_stages(typename Ar::T* x, int s0, int g,
                                          const Tw<typename Ar::T>* __restrict__ W,
                                          const Ar& ar) {
    using T = typename Ar::T;
#pragma unroll
    for (int l = RL - 1; l >= 0; --l) {
        const int h = 1 << (RL - l - 1);
        const Tw<T>* Ws = W + (1 << (s0 + l)) + (g << l);
#pragma unroll
        for (int q = 0; q < (1 << l); ++q) {
            const Tw<T> w = ld_tw(Ws + q);
#pragma unroll
            for (int u = 0; u < h; ++u) {
                const int k = (q << (RL - l)) + u;
                ar.gs(x[k], x[k + h], w.w, w.wq);
            }
        }
    }
}

// One round over all sub-problems of a batch of 2^log_cb vectors of length
// 2^log_len.  ld(v, idx, k) / st(v, idx, val) move element idx of vector v.
template <class Ar, int RL, bool INV, class LD, class ST>
__device__ __forceinline__ void run_round(int log_len, int log_cb, int s0,
                                          const Tw<typename Ar::T>* __restrict__ W,
                                          const Ar& ar, bool zt, LD ld, ST st) {
    using T = typename Ar::T;
    const int d_log = log_len - s0 - RL;
    const int nsub = 1 << (log_cb + log_len - RL);
    for (int sp = threadIdx.x; sp < nsub; sp += blockDim.x) {
        const int v = sp & ((1 << log_cb) - 1);
        const int rest = sp >> log_cb;
        const int j = rest & ((1 << d_log) - 1);
        const int g = rest >> d_log;
        const int base = (g << (d_log + RL)) + j;
        T x[1 << RL];
#pragma unroll
        for (int k = 0; k < (1 << RL); ++k) x[k] = ld(v, base + (k << d_log), k);
        if constexpr (!INV) {
            ct_stages<Ar, RL>(x, s0, g, W, ar, zt);
        } else {
            gs_stages<Ar, RL>(x, s0, g, W, ar);
        }
#pragma unroll
        for (int k = 0; k < (1 << RL); ++k) st(v, base + (k << d_log), x[k]);
    }
}

template <class Ar, bool INV, class LD, class ST>
__device__ __forceinline__ void run_round_rl(int rl, int log_len, int log_cb, int s0,
                                             const Tw<typename Ar::T>* __restrict__ W,
                                             const Ar& ar, bool zt, LD ld, ST st) {
    switch (rl) {
        case 1: run_round<Ar, 1, INV>(log_len, log_cb, s0, W, ar, zt, ld, st); break;
        case 2: run_round<Ar, 2, INV>(log_len, log_cb, s0, W, ar, zt, ld, st); break;
        case 3: run_round<Ar, 3, INV>(log_len, log_cb, s0, W, ar, zt, ld, st); break;
        default: run_round<Ar, 4, INV>(log_len, log_cb, s0, W, ar, zt, ld, st); break;
    }
}

// Apply a two-level inter-pass twiddle w^e = TL[e mod 2^lo] * TH[e >> lo].
template <class Ar>
__device__ __forceinline__ typename Ar::T twiddle2(const Ar& ar, typename Ar::T x, uint32_t e,
                                                   int lo, const Tw<typename Ar::T>* TL,
                                                   const Tw<typename Ar::T>* TH) {
    const auto a = ld_tw(TL + (e & ((1u << lo) - 1)));
    const auto b = ld_tw(TH + (e >> lo));
    return ar.shoup(ar.shoup(x, a.w, a.wq), b.w, b.wq);
}

// ------------------------------------------------------------------ K1
// Forward column pass for one operand (blockIdx.z) and one tile of CB
// columns (blockIdx.x); loops over the K primes reusing the loaded
// coefficients.  ncoef = number of coefficients of the operand; the column
// tail beyond it is the virtual zero pad.  zt_mask bit z says operand z has
// all coefficients in the top half of the rows (rows >= R/2 are zero).
template <class Ar, bool SPLIT16>
__global__ void __launch_bounds__(kColThreads)
k_fwd_col(const PlanDev<Ar> P, const uint32_t* __restrict__ limbs_a, size_t ncoef_a,
          const uint32_t* __restrict__ limbs_b, size_t ncoef_b, typename Ar::T* res_a,
          typename Ar::T* res_b, unsigned zt_mask) {
    using T = typename Ar::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int op = blockIdx.z;
    const uint32_t* __restrict__ limbs = op ? limbs_b : limbs_a;
    const size_t ncoef = op ? ncoef_b : ncoef_a;
    T* res = op ? res_b : res_a;
    const bool zt = ((zt_mask >> op) & 1u) && P.log_r > 0;
    const int log_r = P.log_r, log_c = P.log_c, log_cb = P.log_cb;
    const int R = 1 << log_r, CB = 1 << log_cb;
    const size_t C = (size_t)1 << log_c;
    const size_t n = (size_t)R * C;
    const int c0 = blockIdx.x << log_cb;
    const int rows_loaded = zt ? R / 2 : R;

    T* buf = reinterpret_cast<T*>(smem_raw);
    uint32_t* coef = reinterpret_cast<uint32_t*>(buf + (R << log_cb));

    for (int e = threadIdx.x; e < (rows_loaded << log_cb); e += blockDim.x) {
        const size_t ci = (size_t)(e >> log_cb) * C + c0 + (e & (CB - 1));
        uint32_t val = 0;
        if (ci < ncoef) {
            if constexpr (SPLIT16) {
                val = (__ldg(limbs + (ci >> 1)) >> ((ci & 1) * 16)) & 0xFFFFu;
            } else {
                val = __ldg(limbs + ci);
            }
        }
        coef[e] = val;
    }
    __syncthreads();

    const Sched sc = make_sched(log_r);
    for (int kp = 0; kp < P.K; ++kp) {
        const PrimeDev<Ar>& pr = P.pr[kp];
        const Ar ar = pr.ar;
        T* gout = res + (size_t)kp * n;
        for (int r = 0; r < sc.n; ++r) {
            const bool first = (r == 0), last = (r == sc.n - 1);
            auto ld_coef = [&](int v, int idx, int k) -> T {
                if (zt && k >= 0 && idx >= R / 2) return T(0);
                return (T)coef[(idx << log_cb) + v];
            };
            auto ld_smem = [&](int v, int idx, int) -> T { return buf[swz<T>((idx << log_cb) + v)]; };
            auto st_smem = [&](int v, int idx, T val) { buf[swz<T>((idx << log_cb) + v)] = val; };
            auto st_glob = [&](int v, int idx, T val) {
                const uint32_t c = (uint32_t)(c0 + v);
                const uint32_t e = c * bitrev((uint32_t)idx, log_r);
                gout[(size_t)idx * C + c] = twiddle2(ar, val, e, P.lo, pr.TLf, pr.THf);
            };
            if (first && last) {
                run_round_rl<Ar, false>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRf, ar, zt, ld_coef, st_glob);
            } else if (first) {
                run_round_rl<Ar, false>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRf, ar, zt, ld_coef, st_smem);
            } else if (last) {
                run_round_rl<Ar, false>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRf, ar, false, ld_smem, st_glob);
            } else {
                run_round_rl<Ar, false>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRf, ar, false, ld_smem, st_smem);
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------ K2
// Fused row pass for row blockIdx.x and prime blockIdx.y: forward C-point NTT
// of both rows, pointwise product, inverse C-point NTT, inverse twiddle.
// The result overwrites the A row.  square: B is A.
template <class Ar, int NT>
__global__ void __launch_bounds__(NT)
k_row(const PlanDev<Ar> P, typename Ar::T* res_a, const typename Ar::T* res_b, int square) {
    using T = typename Ar::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int log_r = P.log_r, log_c = P.log_c;
    const int C = 1 << log_c;
    const size_t n = (size_t)C << log_r;
    const int prow = blockIdx.x;
    const int kp = blockIdx.y;
    const PrimeDev<Ar>& pr = P.pr[kp];
    const Ar ar = pr.ar;
    T* ga = res_a + (size_t)kp * n + (size_t)prow * C;
    const T* gb = res_b + (size_t)kp * n + (size_t)prow * C;
    T* bufA = reinterpret_cast<T*>(smem_raw);
    T* bufB = bufA + C;

    for (int i = threadIdx.x; i < C; i += NT) {
        bufA[swz<T>(i)] = ga[i];
        if (!square) bufB[swz<T>(i)] = gb[i];
    }
    __syncthreads();

    const Sched sc = make_sched(log_c);
    auto ldA = [&](int, int idx, int) -> T { return bufA[swz<T>(idx)]; };
    auto stA = [&](int, int idx, T v) { bufA[swz<T>(idx)] = v; };
    auto ldB = [&](int, int idx, int) -> T { return bufB[swz<T>(idx)]; };
    auto stB = [&](int, int idx, T v) { bufB[swz<T>(idx)] = v; };
    const uint32_t k1 = bitrev((uint32_t)prow, log_r);
    auto st_glob = [&](int, int idx, T v) {
        const uint32_t e = (uint32_t)idx * k1;
        ga[idx] = twiddle2(ar, v, e, P.lo, pr.TLi, pr.THi);
    };

    // forward rounds: A fully (all but the last when squaring), B all but the last
    const int a_rounds = square ? sc.n - 1 : sc.n;
    for (int r = 0; r < a_rounds; ++r) {
        run_round_rl<Ar, false>(sc.rl[r], log_c, 0, sc.s0[r], pr.WCf, ar, false, ldA, stA);
        __syncthreads();
    }
    if (!square) {
        for (int r = 0; r < sc.n - 1; ++r) {
            run_round_rl<Ar, false>(sc.rl[r], log_c, 0, sc.s0[r], pr.WCf, ar, false, ldB, stB);
            __syncthreads();
        }
    }

    // fused round: last forward round of B (or A), pointwise product, first
    // inverse round -- one sub-problem stays in registers throughout.
    {
        const int r = sc.n - 1;
        const int rl = sc.rl[r], s0 = sc.s0[r];
        const int d_log = log_c - s0 - rl;
        const int nsub = 1 << (log_c - rl);
        const bool final_round = (sc.n == 1);
        T* src = square ? bufA : bufB;
        for (int sp = threadIdx.x; sp < nsub; sp += NT) {
            const int j = sp & ((1 << d_log) - 1);
            const int g = sp >> d_log;
            const int base = (g << (d_log + rl)) + j;
            T x[16];
#define BW_FUSED_BODY(RL)                                                              \
    {                                                                                  \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) x[k] =                   \
            src[swz<T>(base + (k << d_log))];                                          \
        ct_stages<Ar, RL>(x, s0, g, pr.WCf, ar, false);                                \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) {                        \
            const T xa = ar.red2(x[k]);                                                \
            const T ya = square ? xa : ar.red2(bufA[swz<T>(base + (k << d_log))]);     \
            x[k] = ar.mont(xa, ya);                                                    \
        }                                                                              \
        gs_stages<Ar, RL>(x, s0, g, pr.WCi, ar);                                       \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) {                        \
            const int idx = base + (k << d_log);                                       \
            if (final_round) st_glob(0, idx, x[k]); else bufA[swz<T>(idx)] = x[k];     \
        }                                                                              \
    }
            switch (rl) {
                case 1: BW_FUSED_BODY(1) break;
                case 2: BW_FUSED_BODY(2) break;
                case 3: BW_FUSED_BODY(3) break;
                default: BW_FUSED_BODY(4) break;
            }
#undef BW_FUSED_BODY
        }
        __syncthreads();
    }

    // remaining inverse rounds, last one writes to global with the twiddle
    for (int r = sc.n - 2; r >= 0; --r) {
        if (r == 0) {
            run_round_rl<Ar, true>(sc.rl[r], log_c, 0, sc.s0[r], pr.WCi, ar, false, ldA, st_glob);
        } else {
            run_round_rl<Ar, true>(sc.rl[r], log_c, 0, sc.s0[r], pr.WCi, ar, false, ldA, stA);
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------ K3
// Inverse column pass for prime blockIdx.y, column tile blockIdx.x.  Writes
// fully reduced residues of the cyclic convolution in natural order, in place.
// Block (0,0) also resets the carry ticket for the K4 launch that follows.
template <class Ar>
__global__ void __launch_bounds__(kColThreads)
k_inv_col(const PlanDev<Ar> P, typename Ar::T* res, CarryState* cst) {
    using T = typename Ar::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) cst->counter = 0;
    const int log_r = P.log_r, log_c = P.log_c, log_cb = P.log_cb;
    const int R = 1 << log_r;
    const size_t C = (size_t)1 << log_c;
    const size_t n = (size_t)R * C;
    const int c0 = blockIdx.x << log_cb;
    const int kp = blockIdx.y;
    const PrimeDev<Ar>& pr = P.pr[kp];
    const Ar ar = pr.ar;
    T* g = res + (size_t)kp * n;
    T* buf = reinterpret_cast<T*>(smem_raw);

    auto ld_glob = [&](int v, int idx, int) -> T { return g[(size_t)idx * C + c0 + v]; };
    auto st_glob = [&](int v, int idx, T val) { g[(size_t)idx * C + c0 + v] = ar.red1(val); };
    auto ld_smem = [&](int v, int idx, int) -> T { return buf[swz<T>((idx << log_cb) + v)]; };
    auto st_smem = [&](int v, int idx, T val) { buf[swz<T>((idx << log_cb) + v)] = val; };

    const Sched sc = make_sched(log_r);
    for (int r = sc.n - 1; r >= 0; --r) {
        const bool first = (r == sc.n - 1), last = (r == 0);
        if (first && last) {
            run_round_rl<Ar, true>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRi, ar, false, ld_glob, st_glob);
        } else if (first) {
            run_round_rl<Ar, true>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRi, ar, false, ld_glob, st_smem);
        } else if (last) {
            run_round_rl<Ar, true>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRi, ar, false, ld_smem, st_glob);
        } else {
            run_round_rl<Ar, true>(sc.rl[r], log_r, log_cb, sc.s0[r], pr.WRi, ar, false, ld_smem, st_smem);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ K4
// Garner + carry.  Output word j of the product collects the "digit sum"
// D_j (< 2^96): the coefficient j (32-bit coefficients), or coefficients
// 2j + 2^16 * (2j+1) (16-bit coefficients).  The product is sum D_j 2^(32 j).
//
// Every thread turns its 8 digit sums into 8 words plus a carry-out X
// (< 2^66), computed with carry-in zero.  The true carry into a span of
// words is "X of the span just before it" plus a single bit eps (the sum of
// the words with that carry overflows at most once), and eps obeys
// generate / propagate / kill rules.  So thread- and tile-level carries
// reduce to 1-bit scans: ballots inside a warp, a short loop across warps,
// and a decoupled look-back across tiles.  A tile publishes its carry words
// (the last thread's X) before it waits on anything, then its status, then
// its inclusive eps.  Tiles are claimed in order through an atomic ticket,
// so every tile a CTA waits on is already running.  Every wait is bounded;
// on timeout bit 0 of *err is set and the kernel finishes.  Records are
// written with tag `epoch` and awaited with tag `wait_epoch` (equal except
// under the fault-injection test hook, which makes every wait run out).
//
// Reference: crt_combine_kernel (src/crt_gpu.cu:157-203, 231-276) and the
// three-pass carry (src/carry_prop.cu:8-80) with its host-polled fixup loop
// (src/gpu_ntt.cu:908-924).

// CTA-wide resolution of a 1-bit carry chain.  Each thread has a status
// st: 0 kill, 1 propagate, 2 generate.  chain_prepare publishes per-warp
// aggregates (carry out for carry-in 0 / 1) in s_w and must be followed by a
// __syncthreads(); chain_out gives the CTA carry-out for a carry-in, and
// chain_mine the carry into the calling thread.
struct ChainMasks {
    uint64_t A, B;
};
__device__ __forceinline__ ChainMasks chain_prepare(int st, uint32_t* s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t G = __ballot_sync(0xffffffffu, st == 2);
    const uint32_t Pm = __ballot_sync(0xffffffffu, st == 1);
    ChainMasks m;
    m.A = (uint64_t)(G | Pm);
    m.B = (uint64_t)G;
    if (lane == 0) {
        const uint32_t c0 = (uint32_t)((m.A + m.B) >> 32) & 1u;
        const uint32_t c1 = (uint32_t)((m.A + m.B + 1) >> 32) & 1u;
        s_w[warp] = c0 | (c1 << 1);
    }
    return m;
}
__device__ __forceinline__ uint32_t chain_out(const uint32_t* s_w, uint32_t cin) {
    uint32_t c = cin;
    const int nw = blockDim.x >> 5;
    for (int w = 0; w < nw; ++w) c = (s_w[w] >> c) & 1u;
    return c;
}
__device__ __forceinline__ uint32_t chain_mine(const ChainMasks& m, const uint32_t* s_w,
                                               uint32_t cin) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t ci = cin;
    for (int w = 0; w < warp; ++w) ci = (s_w[w] >> ci) & 1u;
    const uint64_t S = m.A + m.B + ci;
    const uint32_t carries = (uint32_t)(S ^ m.A ^ m.B);
    return (carries >> lane) & 1u;
}

template <class Ar, bool SPLIT16>
__global__ void __launch_bounds__(kCarryThreads)
k_garner_carry(const PlanDev<Ar> P, const typename Ar::T* __restrict__ res,
               uint32_t* __restrict__ out, size_t M, size_t NL, CarryState* cst,
               uint4* __restrict__ rec_x, uint32_t* __restrict__ rec_s, uint32_t epoch,
               uint32_t wait_epoch, uint32_t* __restrict__ err, int spin_limit) {
    using T = typename Ar::T;
    constexpr int E = kCarryWordsPerThread;
    constexpr int TL = kCarryTileWords;
    constexpr int CPW = SPLIT16 ? 2 : 1;  // coefficients per output word
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_w[kCarryThreads / 32];
    __shared__ uint32_t s_lastx[kCarryThreads / 32][3];
    __shared__ uint32_t s_cin[3];
    __shared__ uint32_t s_eps;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(&cst->counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const size_t j0 = (size_t)t * TL + (size_t)tid * E;
    const size_t n = (size_t)1 << P.log_n;

    // ---- Garner: digit sums D[e] < 2^96
    unsigned __int128 D[E];
    uint32_t bad = 0;
    {
        const Ar a1 = P.pr[1].ar;
        const GarnerDev<Ar>& G = P.gar;
        T r[kMaxPrimes][E * CPW];
#pragma unroll
        for (int kp = 0; kp < kMaxPrimes; ++kp)
#pragma unroll
            for (int q = 0; q < E * CPW; ++q) r[kp][q] = 0;
        if (j0 < NL) {
            // 128-bit vector loads of E*CPW consecutive residues per prime
#pragma unroll
            for (int kp = 0; kp < kMaxPrimes; ++kp) {
                if (kp >= P.K) break;
                const uint4* src =
                    reinterpret_cast<const uint4*>(res + (size_t)kp * n + j0 * CPW);
#pragma unroll
                for (int q = 0; q < (E * CPW * (int)sizeof(T)) / 16; ++q) {
                    const uint4 v = __ldg(src + q);
                    if constexpr (sizeof(T) == 8) {
                        r[kp][2 * q] = ((uint64_t)v.y << 32) | v.x;
                        r[kp][2 * q + 1] = ((uint64_t)v.w << 32) | v.z;
                    } else {
                        r[kp][4 * q] = v.x;
                        r[kp][4 * q + 1] = v.y;
                        r[kp][4 * q + 2] = v.z;
                        r[kp][4 * q + 3] = v.w;
                    }
                }
            }
        }
        unsigned __int128 x[E * CPW];
#pragma unroll
        for (int q = 0; q < E * CPW; ++q) {
            const T r0 = r[0][q];
            // k1 = (r1 - r0) * p0^-1 mod p1
            const T r0m1 = a1.red1(a1.shoup(r0, 1, P.pr[1].one_q));
            const T t1 = r[1][q] >= r0m1 ? r[1][q] - r0m1 : r[1][q] + a1.p - r0m1;
            const T k1 = a1.red1(a1.shoup(t1, G.inv1, G.inv1q));
            x[q] = (unsigned __int128)G.p0 * k1 + r0;
            if (P.K == 3) {
                // the third prime is redundant for every supported size: the
                // mixed-radix digit k2 must be 0, otherwise flag an error
                const Ar a2 = P.pr[2].ar;
                const T r0m2 = a2.red1(a2.shoup(r0, 1, P.pr[2].one_q));
                const T y = a2.red1(r0m2 + a2.red1(a2.shoup(k1, G.p0m2, G.p0m2q)));
                const T r2 = r[2][q];
                const T t2 = r2 >= y ? r2 - y : r2 + a2.p - y;
                const T k2 = a2.red1(a2.shoup(t2, G.inv2, G.inv2q));
                bad |= (k2 != 0);
            }
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
            if constexpr (SPLIT16) {
                D[e] = x[2 * e] + (x[2 * e + 1] << 16);
            } else {
                D[e] = x[e];
            }
            bad |= (uint32_t)((D[e] >> 96) != 0);
        }
    }
    if (bad) atomicOr(err, 2u);

    // ---- local carry: words l[0..E) and carry-out X < 2^66
    uint32_t l[E];
    uint32_t X[3];
    {
        unsigned __int128 acc = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            acc += D[e];
            l[e] = (uint32_t)acc;
            acc >>= 32;
        }
        X[0] = (uint32_t)acc;
        X[1] = (uint32_t)(acc >> 32);
        X[2] = (uint32_t)(acc >> 64);
    }

    // ---- the tile's carry words: the last thread's X, published at once
    // (it depends on nothing outside the tile)
    if (tid == kCarryThreads - 1) {
        uint32_t* rx = reinterpret_cast<uint32_t*>(rec_x + t);
        st_relaxed(rx + 0, X[0]);
        st_relaxed(rx + 1, X[1]);
        st_relaxed(rx + 2, X[2]);
        st_release(rx + 3, epoch);
    }

    // ---- predecessor's carry words: shuffle, shared memory, or (thread 0)
    // the previous tile's record
    uint32_t PX[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) PX[q] = __shfl_up_sync(0xffffffffu, X[q], 1);
    if (lane == 31) {
        s_lastx[warp][0] = X[0];
        s_lastx[warp][1] = X[1];
        s_lastx[warp][2] = X[2];
    }
    if (tid == 0) {
        s_cin[0] = s_cin[1] = s_cin[2] = 0;
        if (t > 0) {
            const uint32_t* rx = reinterpret_cast<const uint32_t*>(rec_x + (t - 1));
            int it = 0;
            bool ok = true;
            while (ld_acquire(rx + 3) != wait_epoch) {
                if (++it > spin_limit) {
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
            if (ok) {
                s_cin[0] = ld_relaxed(rx + 0);
                s_cin[1] = ld_relaxed(rx + 1);
                s_cin[2] = ld_relaxed(rx + 2);
            } else {
                atomicOr(err, 1u);
            }
        }
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 3; ++q) PX[q] = warp > 0 ? s_lastx[warp - 1][q] : s_cin[q];
    }

    // ---- S = l + PX and this thread's status
    uint32_t S[E];
    int st;
    {
        uint64_t c = 0;
        uint32_t all = 0xffffffffu;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint64_t s = (uint64_t)l[e] + (e < 3 ? PX[e] : 0u) + c;
            S[e] = (uint32_t)s;
            c = s >> 32;
            all &= S[e];
        }
        st = c ? 2 : (all == 0xffffffffu ? 1 : 0);
    }

    const ChainMasks cm = chain_prepare(st, s_w);
    __syncthreads();

    // ---- tile status, publish, look back (thread 0)
    if (tid == 0) {
        const uint32_t c0 = chain_out(s_w, 0u), c1 = chain_out(s_w, 1u);
        const uint32_t kind = c0 ? 2u : (c1 ? 1u : 0u);
        const uint32_t tag = epoch << 4;
        uint32_t eps_in = 0;
        if (t > 0) {
            st_release(rec_s + t, tag | kind);
            int j = (int)t - 1;
            int it = 0;
            for (;;) {
                const uint32_t v = ld_acquire(rec_s + j);
                if ((v >> 4) != (wait_epoch & 0x0fffffffu)) {
                    if (++it > spin_limit) {
                        atomicOr(err, 1u);
                        eps_in = 0;
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                if (v & 8u) {
                    eps_in = (v >> 2) & 1u;
                    break;
                }
                const uint32_t k = v & 3u;
                if (k != 1u || j == 0) {
                    eps_in = (k == 2u) ? 1u : 0u;
                    break;
                }
                --j;
            }
        }
        const uint32_t eps_out = kind == 2u ? 1u : (kind == 1u ? eps_in : 0u);
        st_release(rec_s + t, tag | 8u | (eps_out << 2) | kind);
        s_eps = eps_in;
    }
    __syncthreads();

    // ---- final words
    const uint32_t mc = chain_mine(cm, s_w, s_eps);
    uint32_t w[E];
    {
        uint64_t c = mc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint64_t s = (uint64_t)S[e] + c;
            w[e] = (uint32_t)s;
            c = s >> 32;
        }
    }
    if (j0 + E <= M && ((reinterpret_cast<uintptr_t>(out + j0) & 15u) == 0)) {
        uint4* o = reinterpret_cast<uint4*>(out + j0);
        o[0] = make_uint4(w[0], w[1], w[2], w[3]);
        o[1] = make_uint4(w[4], w[5], w[6], w[7]);
    } else {
#pragma unroll
        for (int e = 0; e < E; ++e)
            if (j0 + e < M) out[j0 + e] = w[e];
    }
}

}  // namespace bw
