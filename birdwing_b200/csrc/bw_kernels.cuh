// bw_kernels.cuh -- device side of the product pipeline (both prime paths).
//
// A product of two operands is computed as a cyclic convolution of length
// n = 2^log_n = R * C per prime with a 4-step NTT (R rows, C columns,
// element (r, c) = coefficient r*C + c):
//
//   K1 fwd_col   per operand, per tile of CB columns: limb split + virtual
//                zero pad, R-point forward NTT down each column, write.
//   K2 row       per prime, per row p (k1 = bitrev(p)): inter-pass twiddle
//                w_n^(c k1) on load, C-point forward NTT of the A row and the
//                B row, pointwise Montgomery product, C-point inverse NTT,
//                inverse twiddle w_n^(-c k1) n^-1 2^bits, write in place.
//   K3 inv_col   per prime, per column tile: R-point inverse NTT down each
//                column, full reduction, write residues in natural order.
//   K4 garner_carry  per tile of 2048 output words: Garner reconstruction of
//                every coefficient from its K residues, carry generation, and
//                carry propagation across tiles by decoupled look-back.
//
// Forward transforms are Cooley-Tukey with natural-order input and
// bit-reversed output; inverse transforms are Gentleman-Sande with
// bit-reversed input and natural output.  Stage s (m = 2^s groups) uses the
// twiddle table entries W[m .. 2m), W[m + i] = w_{2m}^{bitrev_s(i)}.  Each
// round processes up to 2^RLOG elements per thread in registers (radix 8 or
// 16); rounds exchange data through swizzled shared memory.  Stage twiddles
// are read through L1 (the column pass stages them in shared memory when the
// plan asks for it, BW_PLAN_TW_SMEM).  The inter-pass twiddle
// of a row is split as w_n^(c k1) = F[c mod 2^a] G[c >> a] with per-row
// tables F, G (about 2 sqrt(C) entries) built in shared memory at the start
// of K2, their Shoup companions computed on the device.
//
// The reference runs these stages as separate kernels with separate HBM
// passes: zero_pad (src/zero_pad.cu:3-57), GPU-NTT forward/inverse
// (src/gpu_ntt.cu:577-581,742-747), pointwise_mul_kernel
// (src/gpu_ntt.cu:216-238), crt_combine_kernel (src/crt_gpu.cu:157-276) and the
// three carry kernels (src/carry_prop.cu:8-211).
#pragma once
#include <cuda.h>  // CUtensorMap (the type only; maps are encoded on the host)

#include <cstdint>
#include <type_traits>
#include "bw_arith.cuh"

namespace bw {

// Primes of a plan: 2 or 3, or 6 on the 32-bit path with 64-bit coefficients.
constexpr int kMaxPrimes = 6;
// Primes the digit-sum Garner (16- and 32-bit coefficients) reads.
constexpr int kDigitPrimes = 3;
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
    const Tw<T>* TLf;  // row-level twiddle w_m^e for e < 2^lo (m = R_row * C,
    const Tw<T>* THf;  //   R_row the last column length): w_m^(e 2^lo)
    const Tw<T>* TLi;  // w_m^-e
    const Tw<T>* THi;  // w_m^-(e 2^lo) * n^-1 * 2^bits
    const Tw<T>* WMf;  // three-pass schedule: middle (R2-point) stage twiddles
    const Tw<T>* WMi;
    const Tw<T>* OLf;  // three-pass schedule: outer twiddle w_n^e, e < 2^lo_out
    const Tw<T>* OHf;  //   w_n^(e 2^lo_out)
    Ar ar;
    T one_q;           // floor(2^bits / p): Shoup companion of 1 (x mod p)
    Tw<T> scale;       // n^-1 * 2^bits (single-pass transforms of small products)
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
    uint64_t p01_lo, p01_hi;  // p0 p1 as a 128-bit integer (64-bit coefficients)
    // six primes (32-bit path, 64-bit coefficients): p_j^-1 mod p_i with
    // Shoup companions, pair (i, j < i) at index i (i - 1) / 2 + j
    Tw<T> inv6[15];
};

template <class Ar>
struct PlanDev {
    PrimeDev<Ar> pr[kMaxPrimes];
    GarnerDev<Ar> gar;
    int K;
    int log_n, log_r, log_c, lo;  // lo: split of the row-level twiddle exponent
    int log_cb;                   // outer column tile width CB = 2^log_cb (inverse pass)
    int log_cb1;                  // forward column pass tile width
    int tw_smem_r;                // stage the R-point twiddles in shared memory
    int log_fa;                   // per-row twiddle split a (F has 2^a entries)
    // three-pass schedule (n = R * R2 * C): log_r2 > 0, otherwise 0
    int log_r2, log_cb2, lo_out;
};

// Carry look-back state of one context.
struct CarryState {
    uint32_t counter;   // dynamic tile ticket (reset by K3 before every K4)
    uint32_t pad[3];
};

// One product of a batch (device memory).  Residues of product i live at
// element offset res_off of the bucket's residue arenas (K * n elements in
// each of the A and B arenas).
struct BatchProd {
    const uint32_t* a;
    const uint32_t* b;
    uint32_t* out;
    uint32_t la, lb;       // operand words (out receives la + lb words)
    uint32_t square;       // b is a
    uint32_t pad;
    uint64_t res_off;
    CarryState* cst;       // carry look-back state (4-step buckets)
    uint4* rec_x;
    uint32_t* rec_s;
};

// ------------------------------------------------------------------ helpers

// Shared-memory layouts of a tile: element e lives at e + MUL (e >> SH), one
// or two pad slots after every 2^SH elements (1/16 extra either way).  A
// round's sub-problem reads elements E0 + k 2^D (k < 2^RL, the bits of k clear
// of E0's), whose physical indices are p(E0) + p(k 2^D): for D >= SH (and
// D == 0) that is p(E0) + k S with one stride S = 2^D + MUL 2^(D - SH) per
// round, so an access costs one add instead of a swizzle computation; the
// other rounds compute their offsets.  Each kernel's tile is private, so each
// takes the layout whose strides suit its rounds (a model of the warp's
// accesses, bank by bank):
//   LayRow = e + e/16: conflict-free for 8-byte residues at every stride; for
//     4-byte residues one 2-way conflict per warp access at strides >= 32.
//   e + 2 (e/32), 4-byte column tiles (1-8 columns): conflict-free there.
// (An XOR swizzle, conflict-free, measured more ALU work per access in these
// issue-bound kernels.)
template <int SH, int MUL>
struct Lay {
    static __device__ __forceinline__ int p(int e) { return e + MUL * (e >> SH); }
    static __device__ __forceinline__ bool lin(int D) { return D >= SH || D == 0; }
    static __device__ __forceinline__ int stride(int D) {
        return D >= SH ? (1 << D) + MUL * (1 << (D - SH)) : 1;
    }
    // offset of element k of a sub-problem at round stride D: p(k 2^D)
    template <bool LIN>
    static __device__ __forceinline__ int off(int k, int D, int S) {
        return LIN ? k * S : (k << D) + MUL * ((k << D) >> SH);
    }
};
using LayRow = Lay<4, 1>;
template <typename T>
using LayCol = typename std::conditional<sizeof(T) == 4, Lay<5, 2>, Lay<4, 1>>::type;
// Elements of a padded tile of n logical elements (either layout).
__host__ __device__ constexpr size_t tile_elems(size_t n) { return n + (n >> 4); }

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

// Asynchronous global -> shared copy of one element (cp.async): a tile's
// loads are all issued at once and land while the CTA builds its twiddle
// tables; the issuing thread waits for its own copies with cp_async_wait.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* gsrc) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8, "4- or 8-byte elements");
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    if constexpr (sizeof(T) == 8) {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
    }
}
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Round schedule of a 2^log_len-point transform with rounds of up to RLOG
// stages: the remainder round comes first, where the sub-problem stride is
// largest and shared-memory accesses are conflict-free.  Computed
// arithmetically (no arrays, so nothing goes to local memory).
template <int RLOG>
__host__ __device__ __forceinline__ int sched_rounds(int log_len) {
    return (log_len + RLOG - 1) / RLOG;
}
template <int RLOG>
__host__ __device__ __forceinline__ int sched_rl(int log_len, int r) {
    const int rem = log_len % RLOG;
    return (rem && r == 0) ? rem : RLOG;
}
template <int RLOG>
__host__ __device__ __forceinline__ int sched_s0(int log_len, int r) {
    const int rem = log_len % RLOG;
    return rem ? (r == 0 ? 0 : rem + RLOG * (r - 1)) : RLOG * r;
}

// Twiddle load from shared (TS) or global memory.
template <bool TS, typename T>
__device__ __forceinline__ Tw<T> ld_w(const Tw<T>* p) {
    if constexpr (TS) {
        return *p;
    } else {
        return ld_tw(p);
    }
}

// Two consecutive twiddles (4-byte residues: one 16-byte load; the pair's
// first entry has an even index in a 16-byte-aligned table).
template <bool TS, typename T>
__device__ __forceinline__ void ld_w2(const Tw<T>* p, Tw<T>& a, Tw<T>& b) {
    static_assert(sizeof(T) == 4, "4-byte residues");
    const uint4 v = TS ? *reinterpret_cast<const uint4*>(p)
                       : __ldg(reinterpret_cast<const uint4*>(p));
    a = Tw<T>{v.x, v.y};
    b = Tw<T>{v.z, v.w};
}

// Forward CT stages s0 .. s0+RL-1 on one sub-problem of 2^RL elements that
// belongs to group g of stage s0.  In the first round of a transform (s0 = 0)
// stage 0 has twiddle 1 and inputs in [0, 2p), so its butterflies need no
// multiply; with zt (first round of a zero-padded column) the second half is
// zero and stage 0 just duplicates the first half.
template <class Ar, int RL, bool TS>
__device__ __forceinline__ void ct_stages(typename Ar::T* x, int s0, int g,
                                          const Tw<typename Ar::T>* __restrict__ W,
                                          const Ar& ar, bool zt) {
    using T = typename Ar::T;
#pragma unroll
    for (int l = 0; l < RL; ++l) {
        const int h = 1 << (RL - l - 1);
        if (l == 0 && s0 == 0) {
            if (zt) {
#pragma unroll
                for (int u = 0; u < h; ++u) x[u + h] = x[u];
            } else {
#pragma unroll
                for (int u = 0; u < h; ++u) ar.ct1(x[u], x[u + h]);
            }
            continue;
        }
        const Tw<T>* Ws = W + (1 << (s0 + l)) + (g << l);
        if constexpr (sizeof(T) == 4) {
            if (l > 0) {
                // the level's 2^l twiddles in pairs
#pragma unroll
                for (int q = 0; q < (1 << l); q += 2) {
                    Tw<T> w[2];
                    ld_w2<TS>(Ws + q, w[0], w[1]);
#pragma unroll
                    for (int e = 0; e < 2; ++e)
#pragma unroll
                        for (int u = 0; u < h; ++u) {
                            const int k = ((q + e) << (RL - l)) + u;
                            ar.ct(x[k], x[k + h], w[e].w, w[e].wq);
                        }
                }
                continue;
            }
        }
#pragma unroll
        for (int q = 0; q < (1 << l); ++q) {
            const Tw<T> w = ld_w<TS>(Ws + q);
#pragma unroll
            for (int u = 0; u < h; ++u) {
                const int k = (q << (RL - l)) + u;
                ar.ct(x[k], x[k + h], w.w, w.wq);
            }
        }
    }
}

// Inverse GS stages s0+RL-1 down to s0 (the mirror of ct_stages); stage 0
// has twiddle 1.
template <class Ar, int RL, bool TS>
__device__ __forceinline__ void gs_stages(typename Ar::T* x, int s0, int g,
                                          const Tw<typename Ar::T>* __restrict__ W,
                                          const Ar& ar) {
    using T = typename Ar::T;
#pragma unroll
    for (int l = RL - 1; l >= 0; --l) {
        const int h = 1 << (RL - l - 1);
        if (l == 0 && s0 == 0) {
#pragma unroll
            for (int u = 0; u < h; ++u) ar.gs1(x[u], x[u + h]);
            continue;
        }
        const Tw<T>* Ws = W + (1 << (s0 + l)) + (g << l);
        if constexpr (sizeof(T) == 4) {
            if (l > 0) {
#pragma unroll
                for (int q = 0; q < (1 << l); q += 2) {
                    Tw<T> w[2];
                    ld_w2<TS>(Ws + q, w[0], w[1]);
#pragma unroll
                    for (int e = 0; e < 2; ++e)
#pragma unroll
                        for (int u = 0; u < h; ++u) {
                            const int k = ((q + e) << (RL - l)) + u;
                            ar.gs(x[k], x[k + h], w[e].w, w[e].wq);
                        }
                }
                continue;
            }
        }
#pragma unroll
        for (int q = 0; q < (1 << l); ++q) {
            const Tw<T> w = ld_w<TS>(Ws + q);
#pragma unroll
            for (int u = 0; u < h; ++u) {
                const int k = (q << (RL - l)) + u;
                ar.gs(x[k], x[k + h], w.w, w.wq);
            }
        }
    }
}

// One round over all sub-problems of a batch of 2^log_cb vectors of length
// 2^log_len.  ld(v, idx, p) / st(v, idx, p, val) move element idx of vector v,
// whose shared-memory tile slot is p (tile element (idx << log_cb) + v in
// layout L).  LIN: the round's stride D = d + log_cb lets the slots advance
// by a fixed stride (L::stride); otherwise each offset is computed (L::off).
// FCB >= 0: the round has stride 1 in the vector (d_log = 0) and the batch
// width is 2^FCB, both known at compile time, so that every slot offset is an
// immediate (a tile's stride-1 round; log_cb is then ignored).
template <class Ar, class L, int RL, bool INV, bool TS, bool LIN, int FCB = -1, class LD,
          class ST>
__device__ __forceinline__ void run_round(int log_len, int log_cb_rt, int s0,
                                          const Tw<typename Ar::T>* __restrict__ W,
                                          const Ar& ar, bool zt, LD ld, ST st) {
    using T = typename Ar::T;
    const int log_cb = FCB >= 0 ? FCB : log_cb_rt;
    const int d_log = FCB >= 0 ? 0 : log_len - s0 - RL;
    const int D = d_log + log_cb;
    const int S = L::stride(D);
    const int nsub = 1 << (log_cb + log_len - RL);
    for (int sp = threadIdx.x; sp < nsub; sp += blockDim.x) {
        const int v = sp & ((1 << log_cb) - 1);
        const int rest = sp >> log_cb;
        const int j = rest & ((1 << d_log) - 1);
        const int g = rest >> d_log;
        const int base = (g << (d_log + RL)) + j;
        const int p0 = L::p((base << log_cb) + v);
        T x[1 << RL];
#pragma unroll
        for (int k = 0; k < (1 << RL); ++k)
            x[k] = ld(v, base + (k << d_log), p0 + L::template off<LIN>(k, D, S));
        if constexpr (!INV) {
            ct_stages<Ar, RL, TS>(x, s0, g, W, ar, zt);
        } else {
            gs_stages<Ar, RL, TS>(x, s0, g, W, ar);
        }
#pragma unroll
        for (int k = 0; k < (1 << RL); ++k)
            st(v, base + (k << d_log), p0 + L::template off<LIN>(k, D, S), x[k]);
    }
}

// Dispatch on the round's radix and addressing: only the remainder round (the
// first round of a transform) is narrower than 2^RLOG, so the full radix has
// one instantiation per call site and the narrow ones stay small.  A round
// whose stride the layout steps through linearly adds one stride per slot; a
// stride-1 round of a tile up to 16 vectors wide gets compile-time offsets;
// the others compute their offsets.
template <class Ar, class L, int RLOG, bool INV, bool TS, class LD, class ST>
__device__ __forceinline__ void run_round_rl(int rl, int log_len, int log_cb, int s0,
                                             const Tw<typename Ar::T>* __restrict__ W,
                                             const Ar& ar, bool zt, LD ld, ST st) {
    const int d_log = log_len - s0 - rl;
    const int D = d_log + log_cb;
    if (rl == RLOG) {
        // (4-byte residues only: on the 64-bit path the extra instantiations
        // measured slower, the inverse column pass 0.231 -> 0.247 ms)
        if constexpr (sizeof(typename Ar::T) == 4) {
            if (d_log == 0 && log_cb <= 4) {
                switch (log_cb) {
                    case 0:
                        run_round<Ar, L, RLOG, INV, TS, false, 0>(log_len, 0, s0, W, ar,
                                                                  zt, ld, st);
                        return;
                    case 1:
                        run_round<Ar, L, RLOG, INV, TS, false, 1>(log_len, 1, s0, W, ar,
                                                                  zt, ld, st);
                        return;
                    case 2:
                        run_round<Ar, L, RLOG, INV, TS, false, 2>(log_len, 2, s0, W, ar,
                                                                  zt, ld, st);
                        return;
                    case 3:
                        run_round<Ar, L, RLOG, INV, TS, false, 3>(log_len, 3, s0, W, ar,
                                                                  zt, ld, st);
                        return;
                    default:
                        run_round<Ar, L, RLOG, INV, TS, false, 4>(log_len, 4, s0, W, ar,
                                                                  zt, ld, st);
                        return;
                }
            }
        }
        if (L::lin(D)) {
            run_round<Ar, L, RLOG, INV, TS, true>(log_len, log_cb, s0, W, ar, zt, ld, st);
        } else {
            run_round<Ar, L, RLOG, INV, TS, false>(log_len, log_cb, s0, W, ar, zt, ld, st);
        }
    } else if (rl == 3) {
        if (L::lin(D)) {
            run_round<Ar, L, 3, INV, TS, true>(log_len, log_cb, s0, W, ar, zt, ld, st);
        } else {
            run_round<Ar, L, 3, INV, TS, false>(log_len, log_cb, s0, W, ar, zt, ld, st);
        }
    } else if (rl == 2) {
        run_round<Ar, L, 2, INV, TS, false>(log_len, log_cb, s0, W, ar, zt, ld, st);
    } else {
        run_round<Ar, L, 1, INV, TS, false>(log_len, log_cb, s0, W, ar, zt, ld, st);
    }
}

// Copy a stage twiddle table (2^log_len entries) into shared memory.
template <typename T>
__device__ __forceinline__ void stage_table(Tw<T>* dst, const Tw<T>* src, int log_len) {
    for (int i = threadIdx.x; i < (1 << log_len); i += blockDim.x) dst[i] = ld_tw(src + i);
}

// ------------------------------------------------------------------ K1
// Forward column pass for one operand (blockIdx.z) and one tile of CB
// columns (tile0 + blockIdx.x: a launch may cover a range of tiles, so that
// the pass runs behind a copy-in split by columns); loops over the K primes
// reusing the loaded
// coefficients.  ncoef = number of coefficients of the operand; the column
// tail beyond it is the virtual zero pad.  zt_mask bit z says operand z has
// all coefficients in the top half of the rows (rows >= R/2 are zero).
// W64 (64-bit path): 64-bit coefficients, two words each; ncoef is then the
// operand's word count (an odd count leaves the last coefficient's high word
// zero), and each coefficient enters the transform reduced to [0, 3p).
// PP (64-bit path): the CTA transforms for one prime, kp0, and stages the
// coefficients straight into its residue tile, where the first round runs in
// place like the others; without PP it loops over the K primes and keeps a
// separate copy of the coefficients, which halves the tile width its shared
// memory allows.
template <class Ar, bool SPLIT16, int RLOG, bool TS, bool W64 = false, bool PP = false>
__device__ __forceinline__ void fwd_col_body(const PlanDev<Ar>& P,
                                             const uint32_t* __restrict__ limbs, size_t ncoef,
                                             typename Ar::T* res, bool zt_in, int tile,
                                             unsigned char* smem_raw, int kp0 = 0) {
    static_assert(!PP || (!SPLIT16 && (sizeof(typename Ar::T) == 8 || W64)),
                  "PP: 64-bit path, or 64-bit coefficients on the 32-bit path");
    using T = typename Ar::T;
    const bool zt = zt_in && P.log_r > 0;
    const int log_r = P.log_r, log_c = P.log_c + P.log_r2, log_cb = P.log_cb1;
    const int R = 1 << log_r, CB = 1 << log_cb;
    const size_t C = (size_t)1 << log_c;  // stride between rows (R2 * C columns)
    const size_t n = (size_t)R * C;
    const int c0 = tile << log_cb;
    const int rows_loaded = zt ? R / 2 : R;
    // staged coefficients: 16-bit halves (32-bit path), 32-bit limbs or
    // 64-bit limb pairs (64-bit path)
    using CT = typename std::conditional<
        SPLIT16, uint16_t, typename std::conditional<W64, uint64_t, uint32_t>::type>::type;

    Tw<T>* tws = reinterpret_cast<Tw<T>*>(smem_raw);         // R entries if TS
    T* buf = reinterpret_cast<T*>(smem_raw + (TS ? (size_t)R * sizeof(Tw<T>) : 0));
    // 64-bit coefficients after a 4-byte residue tile start at the next 16-byte
    // boundary (the tile's 17 (R CB / 16) elements may leave it 4 bytes off)
    size_t coef_off = tile_elems((size_t)R << log_cb) * sizeof(T);
    if constexpr (W64 && sizeof(T) == 4) coef_off = (coef_off + 15) & ~(size_t)15;
    CT* coef = reinterpret_cast<CT*>(reinterpret_cast<unsigned char*>(buf) + coef_off);

    if constexpr (SPLIT16) {
        if (CB >= 2) {
            // whole limbs (two 16-bit coefficients each) by cp.async into the
            // u16 tile: limb e of the tile holds its coefficients 2e and
            // 2e + 1, exactly the little-endian u16 layout the first round
            // reads (CB is even and C is even, so every row segment is whole
            // limbs)
            const int hcb = CB >> 1;
            uint32_t* coef32 = reinterpret_cast<uint32_t*>(coef);
            const size_t nlimbs = (ncoef + 1) >> 1;
            for (int e = threadIdx.x; e < rows_loaded * hcb; e += blockDim.x) {
                const size_t li = ((size_t)(e / hcb) * C + c0) / 2 + (e % hcb);
                if (li < nlimbs) {
                    cp_async_elem(coef32 + e, limbs + li);
                } else {
                    coef32[e] = 0;
                }
            }
        } else {
            for (int e = threadIdx.x; e < (rows_loaded << log_cb); e += blockDim.x) {
                const size_t ci = (size_t)(e >> log_cb) * C + c0 + (e & (CB - 1));
                coef[e] = (CT)(ci < ncoef ? (__ldg(limbs + (ci >> 1)) >> ((ci & 1) * 16)) & 0xFFFFu
                                          : 0u);
            }
        }
    } else if constexpr (W64 && PP && sizeof(T) == 4) {
        // 32-bit path, one prime per CTA: each 64-bit coefficient is reduced
        // for this prime on its way into the residue tile (the K CTAs of a
        // tile run side by side, so the operand words come from L2 after the
        // first of them)
        const Ar ar0 = P.pr[kp0].ar;
        const bool al8 = (reinterpret_cast<uintptr_t>(limbs) & 7u) == 0;
        for (int e = threadIdx.x; e < (rows_loaded << log_cb); e += blockDim.x) {
            const size_t wi = 2 * ((size_t)(e >> log_cb) * C + c0 + (e & (CB - 1)));
            uint64_t x = 0;
            if (wi + 1 < ncoef) {
                x = al8 ? __ldg(reinterpret_cast<const unsigned long long*>(limbs + wi))
                        : ((uint64_t)__ldg(limbs + wi + 1) << 32) | __ldg(limbs + wi);
            } else if (wi < ncoef) {
                x = __ldg(limbs + wi);
            }
            buf[LayCol<T>::p(e)] = ar0.reduce64(x);
        }
    } else if (W64 && PP && (reinterpret_cast<uintptr_t>(limbs) & 7u) == 0) {
        // 64-bit coefficients of an 8-byte-aligned operand: one 8-byte copy
        // each into the residue tile (a lone last word: 4 bytes, high word 0)
        for (int e = threadIdx.x; e < (rows_loaded << log_cb); e += blockDim.x) {
            const size_t wi = 2 * ((size_t)(e >> log_cb) * C + c0 + (e & (CB - 1)));
            T* dst = buf + LayCol<T>::p(e);
            if (wi + 1 < ncoef) {
                cp_async_elem(dst, reinterpret_cast<const T*>(limbs + wi));
            } else if (wi < ncoef) {
                uint32_t* d32 = reinterpret_cast<uint32_t*>(dst);
                cp_async_elem(d32, limbs + wi);
                d32[1] = 0;
            } else {
                *dst = 0;
            }
        }
    } else {
        const bool al8 = (reinterpret_cast<uintptr_t>(limbs) & 7u) == 0;
        for (int e = threadIdx.x; e < (rows_loaded << log_cb); e += blockDim.x) {
            const size_t ci = (size_t)(e >> log_cb) * C + c0 + (e & (CB - 1));
            if constexpr (PP) {
                // into the residue tile at the first round's (swizzled) slot
                uint32_t* dst = reinterpret_cast<uint32_t*>(buf + LayCol<T>::p(e));
                const size_t wi = W64 ? 2 * ci : ci;
                if (wi < ncoef) {
                    cp_async_elem(dst, limbs + wi);
                } else {
                    dst[0] = 0;
                }
                if (W64 && wi + 1 < ncoef) {
                    cp_async_elem(dst + 1, limbs + wi + 1);
                } else {
                    dst[1] = 0;
                }
            } else if constexpr (W64) {
                // one 8-byte copy from an 8-byte-aligned operand, else two
                // 4-byte copies (the operand may start at an odd word)
                uint32_t* dst = reinterpret_cast<uint32_t*>(coef + e);
                const size_t wi = 2 * ci;
                if (al8 && wi + 1 < ncoef) {
                    cp_async_elem(reinterpret_cast<uint64_t*>(dst),
                                  reinterpret_cast<const uint64_t*>(limbs + wi));
                } else {
                    if (wi < ncoef) {
                        cp_async_elem(dst, limbs + wi);
                    } else {
                        dst[0] = 0;
                    }
                    if (wi + 1 < ncoef) {
                        cp_async_elem(dst + 1, limbs + wi + 1);
                    } else {
                        dst[1] = 0;
                    }
                }
            } else {
                // 32-bit limbs land in shared memory without passing registers
                if (ci < ncoef) {
                    cp_async_elem(coef + e, limbs + ci);
                } else {
                    coef[e] = 0;
                }
            }
        }
    }
    cp_async_wait();

    const int nr = sched_rounds<RLOG>(log_r);
    for (int kp = PP ? kp0 : 0; kp < (PP ? kp0 + 1 : P.K); ++kp) {
        const PrimeDev<Ar>& pr = P.pr[kp];
        const Ar ar = pr.ar;
        T* gout = res + (size_t)kp * n;
        const Tw<T>* W = pr.WRf;
        if constexpr (TS) {
            if (kp > 0) __syncthreads();
            stage_table(tws, pr.WRf, log_r);
            W = tws;
        }
        __syncthreads();
        for (int r = 0; r < nr; ++r) {
            const bool first = (r == 0), last = (r == nr - 1);
            // first round reads the coefficient tile (zero pad virtual), last
            // round writes to global memory
            auto ld = [&](int v, int idx, int p) -> T {
                if (first) {
                    if (zt && idx >= R / 2) return T(0);
                    if constexpr (W64 && sizeof(T) == 4) {
                        // 32-bit path: the staged 64-bit coefficient reduced
                        // to [0, 2p) for this prime (PP: reduced when staged)
                        if constexpr (PP) {
                            return buf[p];
                        } else {
                            return ar.reduce64(coef[(idx << log_cb) + v]);
                        }
                    } else {
                        T x = PP ? buf[p] : (T)coef[(idx << log_cb) + v];
                        if constexpr (W64) {
                            // a 64-bit coefficient (up to 64p) enters reduced
                            // to [0, 2p), leaving the transform its headroom
                            x = ar.reduce_in(x);
                        }
                        return x;
                    }
                }
                return buf[p];
            };
            auto st = [&](int v, int idx, int p, T val) {
                if (last) {
                    gout[(size_t)idx * C + c0 + v] = val;
                } else {
                    buf[p] = val;
                }
            };
            run_round_rl<Ar, LayCol<T>, RLOG, false, TS>(sched_rl<RLOG>(log_r, r), log_r, log_cb,
                                              sched_s0<RLOG>(log_r, r), W, ar, first && zt, ld,
                                              st);
            __syncthreads();
        }
    }
}

// PP (64-bit path): blockIdx.x = tile * K + prime, so the K CTAs of one tile
// are launched next to each other and run together: the first brings the
// tile's operand words into L2 and the others read them from there (with the
// prime as grid.y, the residue writes of the tiles in between evicted them and
// every prime re-read its operands from DRAM).  Three CTAs per SM (at most 85
// registers; the 64-bit kernels then spill 32-80 bytes to the stack): the
// shared-memory tile allows three, and the 2^28-bit product measured K1 4%
// faster than at two (the inverse pass measured slower with the same bound).
template <class Ar, bool SPLIT16, int RLOG, bool TS, bool W64 = false, bool PP = false>
__global__ void __launch_bounds__(kColThreads, 3)
k_fwd_col(const PlanDev<Ar> P, const uint32_t* __restrict__ limbs_a, size_t ncoef_a,
          const uint32_t* __restrict__ limbs_b, size_t ncoef_b, typename Ar::T* res_a,
          typename Ar::T* res_b, unsigned zt_mask, int tile0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int op = blockIdx.z;
    fwd_col_body<Ar, SPLIT16, RLOG, TS, W64, PP>(P, op ? limbs_b : limbs_a,
                                                 op ? ncoef_b : ncoef_a, op ? res_b : res_a,
                                                 (zt_mask >> op) & 1u,
                                                 tile0 + (int)(PP ? blockIdx.x / P.K : blockIdx.x),
                                                 smem_raw, PP ? (int)(blockIdx.x % P.K) : 0);
}

// batched: blockIdx.z = 2 * product + operand
template <class Ar, bool SPLIT16, int RLOG>
__global__ void __launch_bounds__(kColThreads)
kb_fwd_col(const PlanDev<Ar> P, const BatchProd* __restrict__ D, typename Ar::T* res_a,
           typename Ar::T* res_b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BatchProd d = D[blockIdx.z >> 1];
    const int op = blockIdx.z & 1;
    if (op && d.square) return;
    const size_t ncoef = (size_t)(op ? d.lb : d.la) * (SPLIT16 ? 2 : 1);
    const size_t n = (size_t)1 << P.log_n;
    fwd_col_body<Ar, SPLIT16, RLOG, false>(P, op ? d.b : d.a, ncoef,
                                           (op ? res_b : res_a) + d.res_off, ncoef <= n / 2,
                                           blockIdx.x, smem_raw);
}

// ------------------------------------------------------------------ K2
// One stage of a 16 x 16 register transpose across the 16 lanes of a
// half-warp (four stages, SH = 1, 2, 4, 8): for every register pair (k, k|SH)
// the lane whose bit SH is clear keeps x[k] and trades x[k|SH] for its
// partner's x[k]; the partner trades x[k] for this lane's x[k|SH].
template <int SH, typename T>
__device__ __forceinline__ void shfl_transpose_step(T (&x)[16], int lane) {
    const bool up = (lane & SH) != 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        if (k & SH) continue;
        const T send = up ? x[k] : x[k | SH];
        const T recv = __shfl_xor_sync(0xffffffffu, send, SH);
        x[k] = up ? recv : x[k];
        x[k | SH] = up ? x[k | SH] : recv;
    }
}

// Per-row twiddle tables: F[i] = w^(i k1), G[j] = w^(j 2^a k1) (forward) and
// the inverse pair with n^-1 2^bits folded into Gi.  w^e comes from the
// plan's two-level tables; each entry's Shoup companion is computed here.
template <class Ar>
__device__ __forceinline__ Tw<typename Ar::T> pow_entry(const Ar& ar, uint64_t e, int lo,
                                                        const Tw<typename Ar::T>* TL,
                                                        const Tw<typename Ar::T>* TH) {
    using T = typename Ar::T;
    const auto a = ld_tw(TL + (e & ((1ull << lo) - 1)));
    const auto b = ld_tw(TH + (e >> lo));
    const T w = ar.red1(ar.shoup(a.w, b.w, b.wq));
    return Tw<T>{w, ar.companion(w)};
}

// Fused row pass for row blockIdx.x and prime blockIdx.y: inter-pass twiddle
// on load, forward C-point NTT of both rows, pointwise product, inverse
// C-point NTT, inverse twiddle.  The result overwrites the A row.
// square: B is A.
template <class Ar, int NT, int RLOG, bool SHFL = false>
__device__ __forceinline__ void row_body(const PlanDev<Ar>& P, typename Ar::T* res_a,
                                         const typename Ar::T* res_b, int square, int prow,
                                         int kp, unsigned char* smem_raw) {
    using T = typename Ar::T;
    const int log_c = P.log_c;
    const int C = 1 << log_c;
    const size_t n = (size_t)1 << P.log_n;  // residues per prime
    // rows come in groups of R_row = 2^log_rr: the last column pass's length
    const int log_rr = P.log_r2 ? P.log_r2 : P.log_r;
    const size_t n_row = (size_t)C << log_rr;  // length of the row-level twiddle
    const PrimeDev<Ar>& pr = P.pr[kp];
    const Ar ar = pr.ar;
    T* ga = res_a + (size_t)kp * n + (size_t)prow * C;
    const T* gb = res_b + (size_t)kp * n + (size_t)prow * C;
    const int la = P.log_fa, nf = 1 << la, ng = C >> la;
    Tw<T>* F = reinterpret_cast<Tw<T>*>(smem_raw);
    Tw<T>* G = F + nf;
    Tw<T>* Fi = G + ng;
    Tw<T>* Gi = Fi + nf;
    T* bufA = reinterpret_cast<T*>(Gi + ng);
    T* bufB = bufA + tile_elems(C);

    const uint64_t k1 = bitrev((uint32_t)prow & ((1u << log_rr) - 1), log_rr);
    const uint64_t nmask = n_row - 1;
    // F[i] = w^(i k1), G[j] = w^(j 2^a k1), Fi[i] = w^(-i k1) (forward tables
    // at exponent n - e), Gi[j] = w^(-j 2^a k1) n^-1 2^bits (inverse tables,
    // whose high table carries the scale)
    for (int i = threadIdx.x; i < nf + ng; i += NT) {
        if (i < nf) {
            const uint64_t e = ((uint64_t)i * k1) & nmask;
            F[i] = pow_entry(ar, e, P.lo, pr.TLf, pr.THf);
            Fi[i] = pow_entry(ar, (n_row - e) & nmask, P.lo, pr.TLf, pr.THf);
        } else {
            const uint64_t e = (((uint64_t)(i - nf) << la) * k1) & nmask;
            G[i - nf] = pow_entry(ar, e, P.lo, pr.TLf, pr.THf);
            Gi[i - nf] = pow_entry(ar, e, P.lo, pr.TLi, pr.THi);
        }
    }
    __syncthreads();

    // (loading the rows by cp.async during the table build measured slower:
    // the in-place twiddle then costs one more shared-memory pass)
    for (int i = threadIdx.x; i < C; i += NT) {
        const Tw<T> f = F[i & (nf - 1)], g = G[i >> la];
        bufA[LayRow::p(i)] = ar.mulc(ar.mulc(ga[i], f.w, f.wq), g.w, g.wq);
        if (!square) bufB[LayRow::p(i)] = ar.mulc(ar.mulc(gb[i], f.w, f.wq), g.w, g.wq);
    }
    __syncthreads();

    const int nr = sched_rounds<RLOG>(log_c);
    auto ldA = [&](int, int, int p) -> T { return bufA[p]; };
    auto st_glob = [&](int idx, T v) {
        const Tw<T> f = Fi[idx & (nf - 1)], g = Gi[idx >> la];
        ga[idx] = ar.mulc(ar.mulc(v, f.w, f.wq), g.w, g.wq);
    };

    // the warp-shuffle exchange (BW_PLAN_SHFL_ROWS): 2^12-point rows of the
    // 32-bit path on 256 threads, one radix-16 sub-problem per thread per
    // round; B's stride-16 round hands its outputs to the fused stride-1
    // round through registers (a 16 x 16 transpose inside each half-warp)
    // instead of shared memory
    constexpr bool kShflShape = SHFL && sizeof(T) == 4 && RLOG == 4 && NT == 256;
    const bool shfl = kShflShape && log_c == 12 && !square;

    // forward rounds: A fully (all but the last when squaring), B all but the
    // last (its last round is fused with the product below)
    for (int op = 0; op < (square ? 1 : 2); ++op) {
        T* buf = op ? bufB : bufA;
        const int rounds = (op == 0 && !square) ? nr : nr - 1 - (op == 1 && shfl ? 1 : 0);
        auto ld = [&](int, int, int p) -> T { return buf[p]; };
        auto st = [&](int, int, int p, T v) { buf[p] = v; };
        for (int r = 0; r < rounds; ++r) {
            run_round_rl<Ar, LayRow, RLOG, false, false>(sched_rl<RLOG>(log_c, r), log_c, 0,
                                                 sched_s0<RLOG>(log_c, r), pr.WCf, ar, false,
                                                 ld, st);
            __syncthreads();
        }
    }

    if constexpr (kShflShape) {
        if (shfl) {
            // B's stride-16 round (stages 4-7) from shared memory ...
            const int tid = threadIdx.x, lane = tid & 15, g = tid >> 4;
            const int s_mid = sched_s0<4>(log_c, nr - 2), s_last = sched_s0<4>(log_c, nr - 1);
            const int base = (g << 8) + lane;
            const int p0 = LayRow::p(base), S = LayRow::stride(4);
            T x[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = bufB[p0 + k * S];
            ct_stages<Ar, 4, false>(x, s_mid, g, pr.WCf, ar, false);
            // ... then lane j' of the half-warp takes element 16 j' + m of
            // the group's 256 (held by lane m as its register j')
            shfl_transpose_step<1>(x, lane);
            shfl_transpose_step<2>(x, lane);
            shfl_transpose_step<4>(x, lane);
            shfl_transpose_step<8>(x, lane);
            // the fused round on sub-problem tid (stride 1): stages 8-11,
            // product with A, first inverse stages
            const int pb = LayRow::p(tid << 4);
            ct_stages<Ar, 4, false>(x, s_last, tid, pr.WCf, ar, false);
#pragma unroll
            for (int k = 0; k < 16; ++k)
                x[k] = ar.mont(ar.fwd_to_2p(x[k]), ar.fwd_to_2p(bufA[pb + k]));
            gs_stages<Ar, 4, false>(x, s_last, tid, pr.WCi, ar);
#pragma unroll
            for (int k = 0; k < 16; ++k) bufA[pb + k] = x[k];
            __syncthreads();
        }
    }

    // fused round: last forward round of B (or A), pointwise product, first
    // inverse round -- one sub-problem stays in registers throughout.  The
    // last round of the schedule has stride 1 (d_log = 0), so the slots of a
    // sub-problem are swz(base) + k.
    if (!shfl) {
        const int r = nr - 1;
        const int rl = sched_rl<RLOG>(log_c, r), s0 = sched_s0<RLOG>(log_c, r);
        const int d_log = log_c - s0 - rl;
        const int nsub = 1 << (log_c - rl);
        const bool final_round = (nr == 1);
        T* src = square ? bufA : bufB;
        for (int sp = threadIdx.x; sp < nsub; sp += NT) {
            const int j = sp & ((1 << d_log) - 1);
            const int g = sp >> d_log;
            const int base = (g << (d_log + rl)) + j;
            const int p0 = LayRow::p(base);
            T x[1 << RLOG];
#define BW_FUSED_BODY(RL)                                                              \
    {                                                                                  \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) x[k] = src[p0 + k];     \
        ct_stages<Ar, RL, false>(x, s0, g, pr.WCf, ar, false);                         \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) {                        \
            const T xa = ar.fwd_to_2p(x[k]);                                           \
            const T ya = square ? xa : ar.fwd_to_2p(bufA[p0 + k]);                     \
            x[k] = ar.mont(xa, ya);                                                    \
        }                                                                              \
        gs_stages<Ar, RL, false>(x, s0, g, pr.WCi, ar);                                \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) {                        \
            if (final_round) st_glob(base + k, x[k]); else bufA[p0 + k] = x[k];        \
        }                                                                              \
    }
            if (rl == RLOG) {
                BW_FUSED_BODY(RLOG)
            } else if (rl == 3) {
                BW_FUSED_BODY(3)
            } else if (rl == 2) {
                BW_FUSED_BODY(2)
            } else {
                BW_FUSED_BODY(1)
            }
#undef BW_FUSED_BODY
        }
        __syncthreads();
    }

    // remaining inverse rounds, the last one writes to global with the twiddle
    for (int r = nr - 2; r >= 0; --r) {
        const bool last = (r == 0);
        auto st = [&](int, int idx, int p, T v) {
            if (last) {
                st_glob(idx, v);
            } else {
                bufA[p] = v;
            }
        };
        run_round_rl<Ar, LayRow, RLOG, true, false>(sched_rl<RLOG>(log_c, r), log_c, 0,
                                            sched_s0<RLOG>(log_c, r), pr.WCi, ar, false, ldA, st);
        __syncthreads();
    }
}

template <class Ar, int NT, int RLOG, bool SHFL = false>
__global__ void __launch_bounds__(NT)
k_row(const PlanDev<Ar> P, typename Ar::T* res_a, const typename Ar::T* res_b, int square) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    row_body<Ar, NT, RLOG, SHFL>(P, res_a, res_b, square, blockIdx.x, blockIdx.y, smem_raw);
}

// batched: blockIdx.z = product
template <class Ar, int NT, int RLOG>
__global__ void __launch_bounds__(NT)
kb_row(const PlanDev<Ar> P, const BatchProd* __restrict__ D, typename Ar::T* res_a,
       const typename Ar::T* res_b) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BatchProd d = D[blockIdx.z];
    row_body<Ar, NT, RLOG>(P, res_a + d.res_off, (d.square ? res_a : res_b) + d.res_off,
                           d.square, blockIdx.x, blockIdx.y, smem_raw);
}

// ------------------------------------------------------------------ K1b / K3b
// Middle column pass of the three-pass schedule (n = R * R2 * C).  Sub-matrix
// s (blockIdx.y, k1 = bitrev(s) over R) is the contiguous span
// [s R2 C, (s+1) R2 C) viewed as R2 rows of C; a CTA takes CB2 columns of it
// for one prime and operand (blockIdx.z = operand * K + prime).  Forward: the
// outer twiddle w_n^((i2 C + c) k1) on load, then an R2-point forward NTT.
// Inverse: an R2-point inverse NTT, then w_n^-((i2 C + c) k1) on store.  The
// twiddle is split as w_n^(i2 C k1) * w_n^(c k1), both factors in per-CTA
// tables.
template <class Ar, bool INV>
__global__ void __launch_bounds__(kColThreads)
k_mid_col(const PlanDev<Ar> P, typename Ar::T* res_a, typename Ar::T* res_b) {
    using T = typename Ar::T;
    constexpr int RLOG = 4;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int log_r2 = P.log_r2, log_c = P.log_c, log_cb = P.log_cb2;
    const int R2 = 1 << log_r2, CB = 1 << log_cb;
    const size_t n = (size_t)1 << P.log_n;
    const int s = blockIdx.y;
    const int kp = blockIdx.z % P.K;
    const int op = blockIdx.z / P.K;
    const PrimeDev<Ar>& pr = P.pr[kp];
    const Ar ar = pr.ar;
    T* g = (op ? res_b : res_a) + (size_t)kp * n + ((size_t)s << (log_r2 + log_c));
    const int c0 = blockIdx.x << log_cb;
    Tw<T>* Trow = reinterpret_cast<Tw<T>*>(smem_raw);  // R2 entries
    Tw<T>* Tcol = Trow + R2;                             // CB entries
    T* buf = reinterpret_cast<T*>(Tcol + CB);

    // the tile's loads first: they land while the twiddle tables are built
    for (int e = threadIdx.x; e < (R2 << log_cb); e += blockDim.x)
        cp_async_elem(buf + LayCol<T>::p(e), g + ((size_t)(e >> log_cb) << log_c) + c0 + (e & (CB - 1)));
    const uint64_t k1 = bitrev((uint32_t)s, P.log_r);
    const uint64_t nmask = n - 1;
    for (int i = threadIdx.x; i < R2 + CB; i += blockDim.x) {
        uint64_t e = i < R2 ? (((uint64_t)i << log_c) * k1) & nmask
                            : ((uint64_t)(c0 + i - R2) * k1) & nmask;
        if (INV) e = (n - e) & nmask;
        const Tw<T> t = pow_entry(ar, e, P.lo_out, pr.OLf, pr.OHf);
        if (i < R2) {
            Trow[i] = t;
        } else {
            Tcol[i - R2] = t;
        }
    }
    cp_async_wait();  // this thread's elements
    __syncthreads();

    const int nr = sched_rounds<RLOG>(log_r2);
    if constexpr (!INV) {
        for (int e = threadIdx.x; e < (R2 << log_cb); e += blockDim.x) {
            const int i2 = e >> log_cb, v = e & (CB - 1);
            const Tw<T> a = Tcol[v], b = Trow[i2];
            buf[LayCol<T>::p(e)] = ar.mulc(ar.mulc(buf[LayCol<T>::p(e)], a.w, a.wq), b.w, b.wq);
        }
        __syncthreads();
        for (int r = 0; r < nr; ++r) {
            const bool last = (r == nr - 1);
            auto ld = [&](int, int, int p) -> T { return buf[p]; };
            auto st = [&](int v, int idx, int p, T val) {
                if (last) {
                    g[((size_t)idx << log_c) + c0 + v] = val;
                } else {
                    buf[p] = val;
                }
            };
            run_round_rl<Ar, LayCol<T>, RLOG, false, false>(sched_rl<RLOG>(log_r2, r), log_r2, log_cb,
                                                 sched_s0<RLOG>(log_r2, r), pr.WMf, ar, false,
                                                 ld, st);
            __syncthreads();
        }
    } else {
        for (int r = nr - 1; r >= 0; --r) {
            const bool last = (r == 0);
            auto ld = [&](int, int, int p) -> T { return buf[p]; };
            auto st = [&](int v, int idx, int p, T val) {
                if (last) {
                    const Tw<T> a = Tcol[v], b = Trow[idx];
                    g[((size_t)idx << log_c) + c0 + v] =
                        ar.mulc(ar.mulc(val, a.w, a.wq), b.w, b.wq);
                } else {
                    buf[p] = val;
                }
            };
            run_round_rl<Ar, LayCol<T>, RLOG, true, false>(sched_rl<RLOG>(log_r2, r), log_r2, log_cb,
                                                sched_s0<RLOG>(log_r2, r), pr.WMi, ar, false, ld,
                                                st);
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------ K3
// Inverse column pass for prime blockIdx.y, column tile blockIdx.x.  Writes
// fully reduced residues of the cyclic convolution in natural order, in place.
// Block (0,0) also resets the carry ticket for the K4 launch that follows.
template <class Ar, int RLOG, bool TS>
__device__ __forceinline__ void inv_col_body(const PlanDev<Ar>& P, typename Ar::T* res,
                                             CarryState* cst, int tile, int kp,
                                             unsigned char* smem_raw) {
    using T = typename Ar::T;
    if (tile == 0 && kp == 0 && threadIdx.x == 0) cst->counter = 0;
    const int log_r = P.log_r, log_c = P.log_c + P.log_r2, log_cb = P.log_cb;
    const int R = 1 << log_r;
    const size_t C = (size_t)1 << log_c;
    const size_t n = (size_t)R * C;
    const int c0 = tile << log_cb;
    const PrimeDev<Ar>& pr = P.pr[kp];
    const Ar ar = pr.ar;
    T* g = res + (size_t)kp * n;
    Tw<T>* tws = reinterpret_cast<Tw<T>*>(smem_raw);
    T* buf = reinterpret_cast<T*>(smem_raw + (TS ? (size_t)R * sizeof(Tw<T>) : 0));
    const Tw<T>* W = pr.WRi;
    if constexpr (TS) {
        stage_table(tws, pr.WRi, log_r);
        W = tws;
        __syncthreads();
    }

    // the whole tile in flight at once (cp.async), then every round from
    // shared memory; the last round reduces and writes global memory
    for (int e = threadIdx.x; e < (R << log_cb); e += blockDim.x)
        cp_async_elem(buf + LayCol<T>::p(e), g + (size_t)(e >> log_cb) * C + c0 + (e & ((1 << log_cb) - 1)));
    cp_async_wait();
    __syncthreads();

    const int nr = sched_rounds<RLOG>(log_r);
    for (int r = nr - 1; r >= 0; --r) {
        const bool last = (r == 0);
        auto ld = [&](int, int, int p) -> T { return buf[p]; };
        auto st = [&](int v, int idx, int p, T val) {
            if (last) {
                g[(size_t)idx * C + c0 + v] = ar.inv_out(val);
            } else {
                buf[p] = val;
            }
        };
        run_round_rl<Ar, LayCol<T>, RLOG, true, TS>(sched_rl<RLOG>(log_r, r), log_r, log_cb,
                                         sched_s0<RLOG>(log_r, r), W, ar, false, ld, st);
        __syncthreads();
    }
}

// ------------------------------------------------------------------ K3, TMA form
// The inverse column pass with its tile brought in by the tensor-memory
// accelerator (BW_PLAN_TMA_COLS): one thread issues R / BR box copies
// (cp.async.bulk.tensor.3d, CB columns x BR rows of prime blockIdx.y, no
// multicast) that complete on a shared-memory mbarrier; every thread waits on
// it (bounded).  A tensor copy writes its box densely, so the rounds run on an
// unpadded tile: its stride-1 round (a thread reads 16 consecutive rows of one
// column, rows CB words apart) puts the sub-problems of a warp 16 CB words
// apart, on the same banks.  Padding between boxes cannot spread them: a box
// must land on a 128-byte boundary, so any pad is whole bank cycles.  The
// measured alternative to the per-element cp.async of k_inv_col.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <class Ar, int RLOG>
__global__ void __launch_bounds__(kColThreads)
k_inv_col_tma(const PlanDev<Ar> P, typename Ar::T* res, CarryState* cst,
              const __grid_constant__ CUtensorMap tmap, uint32_t* __restrict__ err,
              int spin_limit) {
    using T = typename Ar::T;
    using L = Lay<4, 0>;  // dense, as the tensor copies write it
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int s_ok;
    const int tile = blockIdx.x, kp = blockIdx.y;
    if (tile == 0 && kp == 0 && threadIdx.x == 0) cst->counter = 0;
    const int log_r = P.log_r, log_c = P.log_c, log_cb = P.log_cb;
    const int R = 1 << log_r, CB = 1 << log_cb;
    const size_t C = (size_t)1 << log_c;
    const size_t n = (size_t)R * C;
    const int c0 = tile << log_cb;
    const PrimeDev<Ar>& pr = P.pr[kp];
    const Ar ar = pr.ar;
    T* g = res + (size_t)kp * n;
    // tensor copies land on 128-byte-aligned shared addresses (the launch
    // gives 128 bytes of slack)
    T* buf = reinterpret_cast<T*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u));
    const int BR = R < 256 ? R : 256;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_ok = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bar, (unsigned)((size_t)R * CB * sizeof(T)));
        for (int i = 0; i < R / BR; ++i)
            tma_load_3d(buf + (size_t)i * BR * CB, &tmap, c0, i * BR, kp, &bar);
    }
    {
        int it = 0;
        while (!mbar_try_wait(&bar, 0u)) {
            if (++it > spin_limit) {
                s_ok = 0;
                atomicOr(err, 1u);
                break;
            }
        }
    }
    __syncthreads();
    if (!s_ok) return;
    const int nr = sched_rounds<RLOG>(log_r);
    for (int r = nr - 1; r >= 0; --r) {
        const bool last = (r == 0);
        auto ld = [&](int, int, int p) -> T { return buf[p]; };
        auto st = [&](int v, int idx, int p, T val) {
            if (last) {
                g[(size_t)idx * C + c0 + v] = ar.inv_out(val);
            } else {
                buf[p] = val;
            }
        };
        run_round_rl<Ar, L, RLOG, true, false>(sched_rl<RLOG>(log_r, r), log_r, log_cb,
                                               sched_s0<RLOG>(log_r, r), pr.WRi, ar, false, ld, st);
        __syncthreads();
    }
}

template <class Ar, int RLOG, bool TS>
__global__ void __launch_bounds__(kColThreads)
k_inv_col(const PlanDev<Ar> P, typename Ar::T* res, CarryState* cst) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    inv_col_body<Ar, RLOG, TS>(P, res, cst, blockIdx.x, blockIdx.y, smem_raw);
}

// batched: blockIdx.z = product
template <class Ar, int RLOG>
__global__ void __launch_bounds__(kColThreads)
kb_inv_col(const PlanDev<Ar> P, const BatchProd* __restrict__ D, typename Ar::T* res_a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const BatchProd d = D[blockIdx.z];
    inv_col_body<Ar, RLOG, false>(P, res_a + d.res_off, d.cst, blockIdx.x, blockIdx.y,
                                  smem_raw);
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

// Garner reconstruction of the E output words starting at word j0: digit
// sums D[e] < 2^96 (one coefficient per word, or two 16-bit ones).  Words at
// or beyond NL read nothing and are zero.  Sets *bad when the redundant
// third prime disagrees or a value reaches 2^96.
// base: this thread's first residue of prime 0 (global memory, or a tile
// staged in shared memory); prime k's residues start pstride elements later.
// valid: the words exist (false: they read as zero).
template <class Ar, bool SPLIT16, int E, bool NC = true>
__device__ __forceinline__ void garner_digits_at(const PlanDev<Ar>& P,
                                                 const typename Ar::T* __restrict__ base,
                                                 size_t pstride, bool valid,
                                                 unsigned __int128 (&D)[E], uint32_t* bad_out) {
    using T = typename Ar::T;
    constexpr int CPW = SPLIT16 ? 2 : 1;
    uint32_t bad = 0;
    {
        const Ar a1 = P.pr[1].ar;
        const GarnerDev<Ar>& G = P.gar;
        T r[kDigitPrimes][E * CPW];
#pragma unroll
        for (int kp = 0; kp < kDigitPrimes; ++kp)
#pragma unroll
            for (int q = 0; q < E * CPW; ++q) r[kp][q] = 0;
        if (valid) {
            // 128-bit vector loads of E*CPW consecutive residues per prime
#pragma unroll
            for (int kp = 0; kp < kDigitPrimes; ++kp) {
                if (kp >= P.K) break;
                const uint4* src = reinterpret_cast<const uint4*>(base + (size_t)kp * pstride);
#pragma unroll
                for (int q = 0; q < (E * CPW * (int)sizeof(T)) / 16; ++q) {
                    // NC: read-only path (residues from an earlier kernel);
                    // plain loads when this kernel wrote them
                    const uint4 v = NC ? __ldg(src + q) : src[q];
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
    *bad_out |= bad;
}

template <class Ar, bool SPLIT16, int E, bool NC = true>
__device__ __forceinline__ void garner_digits(const PlanDev<Ar>& P,
                                              const typename Ar::T* __restrict__ res, size_t n,
                                              size_t j0, size_t NL, unsigned __int128 (&D)[E],
                                              uint32_t* bad_out) {
    garner_digits_at<Ar, SPLIT16, E, NC>(P, res + j0 * (SPLIT16 ? 2 : 1), n, j0 < NL, D,
                                         bad_out);
}

// 64-bit coefficients (three primes): the E output words from word j0 (j0
// even, E/2 coefficients from coefficient j0/2) and the carry-out X.  Each
// coefficient is the full mixed-radix value c = r0 + p0 k1 + p0 p1 k2
// (< p0 p1 p2 < 2^186; the coefficients of a product stay below
// min(na, nb) 2^128 < 2^160, so c2 >= 2^32 flags an error).  The words are
// the low 32 E bits of V = sum_q c_q 2^(64 q), X = V >> 32 E (< 2^96).
// Coefficients at or beyond NL / 2 read nothing and are zero.
template <class Ar, int E, bool NC>
__device__ __forceinline__ void garner3_words_at(const PlanDev<Ar>& P,
                                                 const typename Ar::T* __restrict__ base,
                                                 size_t pstride, bool valid,
                                                 uint32_t (&l)[E], uint32_t (&X)[3],
                                                 uint32_t* bad_out) {
    using T = typename Ar::T;
    static_assert(sizeof(T) == 8 && E % 4 == 0, "64-bit residues, whole 16-byte loads");
    constexpr int Q = E / 2;
    T r[3][Q];
#pragma unroll
    for (int kp = 0; kp < 3; ++kp)
#pragma unroll
        for (int q = 0; q < Q; ++q) r[kp][q] = 0;
    if (valid) {
#pragma unroll
        for (int kp = 0; kp < 3; ++kp) {
            const uint4* src = reinterpret_cast<const uint4*>(base + (size_t)kp * pstride);
#pragma unroll
            for (int h = 0; h < Q / 2; ++h) {
                const uint4 v = NC ? __ldg(src + h) : src[h];
                r[kp][2 * h] = ((uint64_t)v.y << 32) | v.x;
                r[kp][2 * h + 1] = ((uint64_t)v.w << 32) | v.z;
            }
        }
    }
    const Ar a1 = P.pr[1].ar, a2 = P.pr[2].ar;
    const GarnerDev<Ar>& G = P.gar;
    uint32_t bad = 0;
    uint64_t acc0 = 0, acc1 = 0;  // running carry (< 2^96)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const T r0 = r[0][q];
        const T r0m1 = a1.red1(a1.shoup(r0, 1, P.pr[1].one_q));
        const T t1 = r[1][q] >= r0m1 ? r[1][q] - r0m1 : r[1][q] + a1.p - r0m1;
        const T k1 = a1.red1(a1.shoup(t1, G.inv1, G.inv1q));
        const T r0m2 = a2.red1(a2.shoup(r0, 1, P.pr[2].one_q));
        const T y = a2.red1(r0m2 + a2.red1(a2.shoup(k1, G.p0m2, G.p0m2q)));
        const T r2 = r[2][q];
        const T t2 = r2 >= y ? r2 - y : r2 + a2.p - y;
        const T k2 = a2.red1(a2.shoup(t2, G.inv2, G.inv2q));
        // c = (r0 + p0 k1) + p01_lo k2 + (p01_hi k2) 2^64
        const unsigned __int128 lo =
            (unsigned __int128)G.p0 * k1 + r0 + (unsigned __int128)G.p01_lo * k2;  // < 2^127
        const unsigned __int128 hi = (lo >> 64) + (unsigned __int128)G.p01_hi * k2;
        const uint64_t c0 = (uint64_t)lo, c1 = (uint64_t)hi, c2 = (uint64_t)(hi >> 64);
        bad |= (uint32_t)((c2 >> 32) != 0);
        // add c to the running carry; emit 64 bits; shift
        const unsigned __int128 s0 = (unsigned __int128)acc0 + c0;
        l[2 * q] = (uint32_t)s0;
        l[2 * q + 1] = (uint32_t)((uint64_t)s0 >> 32);
        const unsigned __int128 s1 = (unsigned __int128)acc1 + c1 + (uint64_t)(s0 >> 64);
        acc0 = (uint64_t)s1;
        acc1 = c2 + (uint64_t)(s1 >> 64);
    }
    X[0] = (uint32_t)acc0;
    X[1] = (uint32_t)(acc0 >> 32);
    X[2] = (uint32_t)acc1;
    bad |= (uint32_t)((acc1 >> 32) != 0);
    *bad_out |= bad;
}

// Six primes below 2^30 (32-bit path, 64-bit coefficients): the same words
// and carry-out as garner3_words_at.  The primes ascend, so a digit k_j
// (< p_j) is already below every later prime.  Mixed radix: k_0 = r_0 and
// k_i = (...((r_i - k_0) p_0^-1 - k_1) p_1^-1 ... - k_(i-1)) p_(i-1)^-1 mod p_i;
// c = k_0 + p_0 (k_1 + p_1 (k_2 + p_2 (k_3 + p_3 (k_4 + p_4 k_5)))) < P < 2^178.
// A product's coefficients stay below min(na, nb) 2^128 <= 2^150, so a top
// word c2 >= 2^32 flags an error (residues that disagree give a c spread over
// [0, P)).
template <class Ar, int E, bool NC>
__device__ __forceinline__ void garner6_words_at(const PlanDev<Ar>& P,
                                                 const uint32_t* __restrict__ base,
                                                 size_t pstride, bool valid, uint32_t (&l)[E],
                                                 uint32_t (&X)[3], uint32_t* bad_out) {
    constexpr int Q = E / 2;
    static_assert(Q % 4 == 0, "whole 16-byte loads");
    uint32_t r[6][Q];
#pragma unroll
    for (int kp = 0; kp < 6; ++kp)
#pragma unroll
        for (int q = 0; q < Q; ++q) r[kp][q] = 0;
    if (valid) {
#pragma unroll
        for (int kp = 0; kp < 6; ++kp) {
            const uint4* src = reinterpret_cast<const uint4*>(base + (size_t)kp * pstride);
#pragma unroll
            for (int h = 0; h < Q / 4; ++h) {
                const uint4 v = NC ? __ldg(src + h) : src[h];
                r[kp][4 * h] = v.x;
                r[kp][4 * h + 1] = v.y;
                r[kp][4 * h + 2] = v.z;
                r[kp][4 * h + 3] = v.w;
            }
        }
    }
    const GarnerDev<Ar>& G = P.gar;
    uint32_t bad = 0;
    uint64_t acc0 = 0, acc1 = 0;  // running carry (< 2^96)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        uint32_t k[6];
        k[0] = r[0][q];
#pragma unroll
        for (int i = 1; i < 6; ++i) {
            const Ar ai = P.pr[i].ar;
            // t stays in [0, 2p_i): t - k_j + p_i < 3p_i < 2^32 is a valid
            // Shoup input, and only the digit itself is reduced to [0, p_i)
            uint32_t t = r[i][q];
#pragma unroll
            for (int j = 0; j < i; ++j) {
                const Tw<uint32_t> iv = G.inv6[i * (i - 1) / 2 + j];
                t = ai.shoup(t - k[j] + ai.p, iv.w, iv.wq);  // k_j < p_j < p_i
            }
            k[i] = ai.red1(t);
        }
        // Horner in 32-bit limbs, each step a chain of 32 x 32 + 64-bit
        // multiply-adds: (k5 p4 + k4) (2 limbs), times p3 plus k3 (3), ...,
        // times p0 plus k0 (6 limbs, < 2^178)
        uint32_t w[6];
        {
            const uint64_t t = (uint64_t)k[5] * P.pr[4].ar.p + k[4];
            w[0] = (uint32_t)t;
            w[1] = (uint32_t)(t >> 32);
        }
#pragma unroll
        for (int st = 0; st < 4; ++st) {
            const uint32_t pm = P.pr[3 - st].ar.p;
            uint64_t t = k[3 - st];
#pragma unroll
            for (int i = 0; i < 2 + st; ++i) {
                t = (uint64_t)w[i] * pm + t;
                w[i] = (uint32_t)t;
                t >>= 32;
            }
            w[2 + st] = (uint32_t)t;
        }
        const uint64_t c0 = ((uint64_t)w[1] << 32) | w[0];
        const uint64_t c1 = ((uint64_t)w[3] << 32) | w[2];
        const uint64_t c2 = ((uint64_t)w[5] << 32) | w[4];
        bad |= (uint32_t)((c2 >> 32) != 0);
        const unsigned __int128 s0 = (unsigned __int128)acc0 + c0;
        l[2 * q] = (uint32_t)s0;
        l[2 * q + 1] = (uint32_t)((uint64_t)s0 >> 32);
        const unsigned __int128 s1 = (unsigned __int128)acc1 + c1 + (uint64_t)(s0 >> 64);
        acc0 = (uint64_t)s1;
        acc1 = c2 + (uint64_t)(s1 >> 64);
    }
    X[0] = (uint32_t)acc0;
    X[1] = (uint32_t)(acc0 >> 32);
    X[2] = (uint32_t)acc1;
    bad |= (uint32_t)((acc1 >> 32) != 0);
    *bad_out |= bad;
}

// 64-bit coefficients: three 58-bit primes (64-bit path) or six 30-bit
// primes (32-bit path).
template <class Ar, int E, bool NC = true>
__device__ __forceinline__ void garner_words_w64_at(const PlanDev<Ar>& P,
                                                    const typename Ar::T* __restrict__ base,
                                                    size_t pstride, bool valid,
                                                    uint32_t (&l)[E], uint32_t (&X)[3],
                                                    uint32_t* bad_out) {
    if constexpr (sizeof(typename Ar::T) == 4) {
        garner6_words_at<Ar, E, NC>(P, base, pstride, valid, l, X, bad_out);
    } else {
        garner3_words_at<Ar, E, NC>(P, base, pstride, valid, l, X, bad_out);
    }
}

template <class Ar, int E, bool NC = true>
__device__ __forceinline__ void garner_words_w64(const PlanDev<Ar>& P,
                                                 const typename Ar::T* __restrict__ res,
                                                 size_t n, size_t j0, size_t NL,
                                                 uint32_t (&l)[E], uint32_t (&X)[3],
                                                 uint32_t* bad_out) {
    garner_words_w64_at<Ar, E, NC>(P, res + j0 / 2, n, j0 < NL, l, X, bad_out);
}

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

// Shared memory of one tile's carry resolution.
struct CarryShared {
    uint32_t w[kCarryThreads / 32];
    uint32_t lastx[kCarryThreads / 32][3];
    uint32_t cin[3];
    uint32_t eps;
};

// Tile t's carry, given every thread's 8 words l (digit sums added with
// carry-in zero) and carry-out X: publish the tile's carry words, take the
// predecessor's, resolve the 1-bit carry chain inside the tile, publish the
// tile status and look back across tiles, then write the final words.  Every
// thread of the CTA calls it; it returns after its last barrier.
__device__ __forceinline__ void carry_finish_tile(
    uint32_t t, size_t j0, const uint32_t (&l)[kCarryWordsPerThread], const uint32_t (&X)[3],
    uint32_t* __restrict__ out, size_t M, uint4* __restrict__ rec_x,
    uint32_t* __restrict__ rec_s, uint32_t epoch, uint32_t wait_epoch,
    uint32_t* __restrict__ err, int spin_limit, CarryShared& sh) {
    constexpr int E = kCarryWordsPerThread;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

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
        sh.lastx[warp][0] = X[0];
        sh.lastx[warp][1] = X[1];
        sh.lastx[warp][2] = X[2];
    }
    if (tid == 0) {
        sh.cin[0] = sh.cin[1] = sh.cin[2] = 0;
        if (t > 0) {
            const uint32_t* rx = reinterpret_cast<const uint32_t*>(rec_x + (t - 1));
            int it = 0;
            bool ok = true;
            while (ld_acquire(rx + 3) != wait_epoch) {
                if (++it > spin_limit) {
                    ok = false;
                    break;
                }
                __nanosleep(32);
            }
            if (ok) {
                sh.cin[0] = ld_relaxed(rx + 0);
                sh.cin[1] = ld_relaxed(rx + 1);
                sh.cin[2] = ld_relaxed(rx + 2);
            } else {
                atomicOr(err, 1u);
            }
        }
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 3; ++q) PX[q] = warp > 0 ? sh.lastx[warp - 1][q] : sh.cin[q];
    }

    // ---- S = l + PX and this thread's status
    uint32_t S[E];
    int st;
    {
        uint64_t c = 0;
        uint32_t all = 0xffffffffu;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint64_t sum = (uint64_t)l[e] + (e < 3 ? PX[e] : 0u) + c;
            S[e] = (uint32_t)sum;
            c = sum >> 32;
            all &= S[e];
        }
        st = c ? 2 : (all == 0xffffffffu ? 1 : 0);
    }

    const ChainMasks cm = chain_prepare(st, sh.w);
    __syncthreads();

    // ---- tile status, publish, look back (thread 0)
    if (tid == 0) {
        const uint32_t c0 = chain_out(sh.w, 0u), c1 = chain_out(sh.w, 1u);
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
                    __nanosleep(32);
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
        sh.eps = eps_in;
    }
    __syncthreads();

    // ---- final words
    const uint32_t mc = chain_mine(cm, sh.w, sh.eps);
    uint32_t w[E];
    {
        uint64_t c = mc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint64_t sum = (uint64_t)S[e] + c;
            w[e] = (uint32_t)sum;
            c = sum >> 32;
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

// Words l and carry-out X of E = 8 output words from digit sums (16- and
// 32-bit coefficients) or full coefficients (64-bit), read from `base` (this
// thread's first residue of prime 0, primes pstride apart; global memory or a
// shared-memory tile).
template <class Ar, bool SPLIT16, bool W64, bool NC>
__device__ __forceinline__ void garner_local(const PlanDev<Ar>& P,
                                             const typename Ar::T* __restrict__ base,
                                             size_t pstride, bool valid,
                                             uint32_t (&l)[kCarryWordsPerThread],
                                             uint32_t (&X)[3], uint32_t* bad) {
    constexpr int E = kCarryWordsPerThread;
    if constexpr (W64) {
        garner_words_w64_at<Ar, E, NC>(P, base, pstride, valid, l, X, bad);
    } else {
        unsigned __int128 D[E];
        garner_digits_at<Ar, SPLIT16, E, NC>(P, base, pstride, valid, D, bad);
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
}

// Residue elements of one word of output: two 16-bit coefficients, one 32-bit
// coefficient, or half a 64-bit coefficient.
template <bool SPLIT16, bool W64>
__host__ __device__ constexpr size_t elems_per_word2() {
    return SPLIT16 ? 4 : W64 ? 1 : 2;  // in halves: x2 of the element count
}

template <class Ar, bool SPLIT16, bool W64 = false>
__device__ __forceinline__ void garner_carry_body(
    const PlanDev<Ar>& P, const typename Ar::T* __restrict__ res, uint32_t* __restrict__ out,
    size_t M, size_t NL, CarryState* cst, uint4* __restrict__ rec_x,
    uint32_t* __restrict__ rec_s, uint32_t epoch, uint32_t wait_epoch,
    uint32_t* __restrict__ err, int spin_limit) {
    constexpr int E = kCarryWordsPerThread;
    constexpr int TL = kCarryTileWords;
    __shared__ uint32_t s_tile;
    __shared__ CarryShared sh;

    const int tid = threadIdx.x;
    if (tid == 0) s_tile = atomicAdd(&cst->counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const size_t j0 = (size_t)t * TL + (size_t)tid * E;
    const size_t n = (size_t)1 << P.log_n;

    uint32_t l[E];
    uint32_t X[3];
    uint32_t bad = 0;
    garner_local<Ar, SPLIT16, W64, true>(P, res + j0 * elems_per_word2<SPLIT16, W64>() / 2, n,
                                         j0 < NL, l, X, &bad);
    if (bad) atomicOr(err, 2u);
    carry_finish_tile(t, j0, l, X, out, M, rec_x, rec_s, epoch, wait_epoch, err, spin_limit, sh);
}

// K4 without waits (single products).  The look-back form above keeps every
// CTA of a tile waiting on its predecessor's records: two or three dependent
// L2 round trips per tile with the whole CTA at a barrier.  Here the 1-bit
// tile carry is left out of the first pass instead: k_carry_bounds has
// already published every tile boundary's carry words X, so tile t writes its
// words as if the carry bit eps into it were 0 and records its kind -- the
// carry bit it passes on for eps = 0 and for eps = 1 (kill: 0/0, propagate:
// 0/1, generate: 1/1).  k_carry_fix then scans the kinds (eps into tile 0 is
// 0) and adds 1 at the first word of each tile whose eps is 1, rippling
// inside the tile (a tile that propagates passes the carry on through the
// next tile's own eps).  For operands of random words no tile but an
// all-ones span generates or propagates, so the fix pass writes nothing.
template <class Ar, bool SPLIT16, bool W64 = false>
__global__ void __launch_bounds__(kCarryThreads, 4)
k_garner_words(const PlanDev<Ar> P, const typename Ar::T* __restrict__ res,
               uint32_t* __restrict__ out, size_t M, size_t NL,
               const uint4* __restrict__ rec_x, uint32_t* __restrict__ kinds,
               uint32_t* __restrict__ err) {
    constexpr int E = kCarryWordsPerThread;
    constexpr int TL = kCarryTileWords;
    __shared__ CarryShared sh;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t t = blockIdx.x;
    const size_t j0 = (size_t)t * TL + (size_t)tid * E;
    const size_t n = (size_t)1 << P.log_n;
    if (tid == 0) {
        // the previous tile's boundary carry words, from the pre-pass
        uint4 px = make_uint4(0, 0, 0, 0);
        if (t > 0) px = __ldcg(rec_x + (t - 1));
        sh.cin[0] = px.x;
        sh.cin[1] = px.y;
        sh.cin[2] = px.z;
    }
    uint32_t l[E];
    uint32_t X[3];
    uint32_t bad = 0;
    garner_local<Ar, SPLIT16, W64, true>(P, res + j0 * elems_per_word2<SPLIT16, W64>() / 2, n,
                                         j0 < NL, l, X, &bad);
    if (bad) atomicOr(err, 2u);
    uint32_t PX[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) PX[q] = __shfl_up_sync(0xffffffffu, X[q], 1);
    if (lane == 31) {
        sh.lastx[warp][0] = X[0];
        sh.lastx[warp][1] = X[1];
        sh.lastx[warp][2] = X[2];
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 3; ++q) PX[q] = warp > 0 ? sh.lastx[warp - 1][q] : sh.cin[q];
    }
    uint32_t S[E];
    int st;
    {
        uint64_t c = 0;
        uint32_t all = 0xffffffffu;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint64_t sum = (uint64_t)l[e] + (e < 3 ? PX[e] : 0u) + c;
            S[e] = (uint32_t)sum;
            c = sum >> 32;
            all &= S[e];
        }
        st = c ? 2 : (all == 0xffffffffu ? 1 : 0);
    }
    const ChainMasks cm = chain_prepare(st, sh.w);
    __syncthreads();
    if (tid == 0) {
        const uint32_t c0 = chain_out(sh.w, 0u), c1 = chain_out(sh.w, 1u);
        kinds[t] = c0 | (c1 << 1);
    }
    const uint32_t mc = chain_mine(cm, sh.w, 0u);
    uint32_t w[E];
    {
        uint64_t c = mc;
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const uint64_t sum = (uint64_t)S[e] + c;
            w[e] = (uint32_t)sum;
            c = sum >> 32;
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

// One CTA: the carry bit into every tile from the kinds k_garner_words left
// (bit 0: carry out for carry-in 0, bit 1: for carry-in 1), then +1 at the
// first word of every tile whose carry-in is 1, rippling inside the tile.
// Each thread takes a contiguous run of tiles; a run passes on a constant
// (its last non-propagating tile's carry) or its own carry-in, and a scan over
// the runs in shared memory gives each run its carry-in.
constexpr int kFixThreads = 1024;
static __global__ void __launch_bounds__(kFixThreads)
k_carry_fix(const uint32_t* __restrict__ kinds, uint32_t ntiles, uint32_t* __restrict__ out,
            size_t M) {
    __shared__ uint32_t s_f[kFixThreads];  // 0, 1: constant carry out; 2: passes carry-in
    const int tid = threadIdx.x;
    const uint32_t per = (ntiles + kFixThreads - 1) / kFixThreads;
    const uint32_t t0 = min(ntiles, (uint32_t)tid * per), t1 = min(ntiles, t0 + per);
    uint32_t f = 2;
    for (uint32_t t = t0; t < t1; ++t) {
        const uint32_t k = __ldcg(kinds + t);
        if (k == 0u || k == 3u) f = k & 1u;  // kill / generate: a constant
    }
    s_f[tid] = f;
    __syncthreads();
    // inclusive scan of "the latest constant": combine(a, b) = b unless b
    // passes its carry-in
    for (int d = 1; d < kFixThreads; d <<= 1) {
        const uint32_t a = tid >= d ? s_f[tid - d] : 2u;
        __syncthreads();
        if (s_f[tid] == 2u) s_f[tid] = a;
        __syncthreads();
    }
    uint32_t eps = tid > 0 ? s_f[tid - 1] : 0u;
    if (eps == 2u) eps = 0u;  // nothing before this run sets it: carry-in 0
    for (uint32_t t = t0; t < t1; ++t) {
        const uint32_t k = __ldcg(kinds + t);
        if (eps) {
            const size_t beg = (size_t)t * kCarryTileWords;
            const size_t end = min(M, beg + kCarryTileWords);
            if (k == 2u) {
                // a propagating tile's words are all ones: with the carry in
                // they all become zero (and the carry passes on)
                for (size_t i = beg; i < end; ++i) out[i] = 0u;
            } else {
                for (size_t i = beg; i < end; ++i) {
                    const uint32_t v = out[i] + 1u;
                    out[i] = v;
                    if (v != 0u) break;
                }
            }
        }
        eps = (k >> eps) & 1u;
    }
}

// Carry words of the last thread of every tile but the last (its 8 words'
// carry-out with carry-in zero), published under `epoch` before K4 runs.
// K4 tile t then finds tile t-1's record ready and waits only on the 1-bit
// look-back, not on its predecessor's Garner phase.  One thread per tile.
template <class Ar, bool SPLIT16, bool W64 = false>
__global__ void __launch_bounds__(256)
k_carry_bounds(const PlanDev<Ar> P, const typename Ar::T* __restrict__ res, size_t NL,
               uint4* __restrict__ rec_x, uint32_t ntiles, uint32_t epoch) {
    constexpr int E = kCarryWordsPerThread;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t + 1 >= ntiles) return;
    const size_t n = (size_t)1 << P.log_n;
    const size_t j0 = (size_t)(t + 1) * kCarryTileWords - E;
    uint32_t X[3];
    uint32_t bad = 0;  // the tile's own pass reports reconstruction errors
    if constexpr (W64) {
        uint32_t l[E];
        garner_words_w64<Ar, E>(P, res, n, j0, NL, l, X, &bad);
    } else {
        unsigned __int128 D[E];
        garner_digits<Ar, SPLIT16, E>(P, res, n, j0, NL, D, &bad);
        unsigned __int128 acc = 0;
#pragma unroll
        for (int e = 0; e < E; ++e) acc = (acc + D[e]) >> 32;
        X[0] = (uint32_t)acc;
        X[1] = (uint32_t)(acc >> 32);
        X[2] = (uint32_t)(acc >> 64);
    }
    uint32_t* rx = reinterpret_cast<uint32_t*>(rec_x + t);
    st_relaxed(rx + 0, X[0]);
    st_relaxed(rx + 1, X[1]);
    st_relaxed(rx + 2, X[2]);
    st_release(rx + 3, epoch);
}

// Four CTAs per SM (at most 64 registers): the tile's barriers and its
// one-bit look-back leave warps idle, which more resident CTAs cover
// (measured 12% faster than three).
template <class Ar, bool SPLIT16, bool W64 = false>
__global__ void __launch_bounds__(kCarryThreads, 4)
k_garner_carry(const PlanDev<Ar> P, const typename Ar::T* __restrict__ res,
               uint32_t* __restrict__ out, size_t M, size_t NL, CarryState* cst,
               uint4* __restrict__ rec_x, uint32_t* __restrict__ rec_s, uint32_t epoch,
               uint32_t wait_epoch, uint32_t* __restrict__ err, int spin_limit) {
    garner_carry_body<Ar, SPLIT16, W64>(P, res, out, M, NL, cst, rec_x, rec_s, epoch,
                                        wait_epoch, err, spin_limit);
}

// batched: blockIdx.y = product
template <class Ar, bool SPLIT16>
__global__ void __launch_bounds__(kCarryThreads, 4)
kb_garner_carry(const PlanDev<Ar> P, const BatchProd* __restrict__ D,
                const typename Ar::T* __restrict__ res_a, uint32_t epoch, uint32_t wait_epoch,
                uint32_t* __restrict__ err, int spin_limit) {
    const BatchProd d = D[blockIdx.y];
    const size_t NL = ((size_t)1 << P.log_n) / (SPLIT16 ? 2 : 1);
    garner_carry_body<Ar, SPLIT16>(P, res_a + d.res_off, d.out, (size_t)d.la + d.lb, NL, d.cst,
                                   d.rec_x, d.rec_s, epoch, wait_epoch, err, spin_limit);
}

// ------------------------------------------------------------------ small products
// One CTA computes a whole product whose n-point transform fits in shared
// memory (a batch bucket of equal n, blockIdx.x = product): for each prime
// the forward transforms of both operands, the pointwise product and the
// inverse transform run in shared memory (stage twiddles pr.WCf / pr.WCi of
// length n, scale pr.scale = n^-1 2^bits), the residues go to a per-product
// global scratch (L2-resident at these sizes); then Garner + carry over the
// product's words in tiles of NT*8 words, the carry handed from tile to tile
// inside the CTA, so no look-back is needed.
// Register bounds: 64-bit residues run radix-8 rounds in 64 registers (four
// 256-thread CTAs per SM; radix 16 took 128, two per SM, 12.5% warps
// active); 32-bit residues get at most 128 (unbounded they took 185, one
// 256-thread CTA per SM).
template <class Ar>
constexpr int ks_min_blocks(int nt) {
    return sizeof(typename Ar::T) == 8 ? 1024 / nt : 512 / nt;
}
template <class Ar, bool SPLIT16, int NT>
__device__ __forceinline__ void ks_product_body(const PlanDev<Ar>& P, const BatchProd& d,
                                                typename Ar::T* scratch,
                                                uint32_t* __restrict__ err,
                                                unsigned char* smem_raw) {
    using T = typename Ar::T;
    constexpr int RLOG = sizeof(T) == 8 ? 3 : 4;
    constexpr int E = kCarryWordsPerThread;
    constexpr int CPW = SPLIT16 ? 2 : 1;
    __shared__ uint32_t s_w[NT / 32];
    __shared__ uint32_t s_lastx[NT / 32][3];
    __shared__ uint32_t s_cin[3];
    __shared__ uint32_t s_eps;
    const int log_n = P.log_n;
    const int n = 1 << log_n;
    T* bufA = reinterpret_cast<T*>(smem_raw);
    T* bufB = bufA + tile_elems(n);
    T* res = scratch + d.res_off;
    const size_t nca = (size_t)d.la * CPW, ncb = (size_t)d.lb * CPW;
    const int sq = d.square;
    const int nr = sched_rounds<RLOG>(log_n);
    auto coef = [&](const uint32_t* src, size_t nc, int i) -> T {
        if ((size_t)i >= nc) return T(0);
        if constexpr (SPLIT16) {
            return (T)((__ldg(src + (i >> 1)) >> ((i & 1) * 16)) & 0xFFFFu);
        } else {
            return (T)__ldg(src + i);
        }
    };
    auto ldA = [&](int, int, int p) -> T { return bufA[p]; };

    for (int kp = 0; kp < P.K; ++kp) {
        const PrimeDev<Ar>& pr = P.pr[kp];
        const Ar ar = pr.ar;
        const Tw<T> sc = pr.scale;
        auto st_res = [&](int idx, T v) {
            res[(size_t)kp * n + idx] = ar.red1(ar.shoup(v, sc.w, sc.wq));
        };
        for (int i = threadIdx.x; i < n; i += NT) {
            bufA[LayRow::p(i)] = coef(d.a, nca, i);
            if (!sq) bufB[LayRow::p(i)] = coef(d.b, ncb, i);
        }
        __syncthreads();
        for (int op = 0; op < (sq ? 1 : 2); ++op) {
            T* buf = op ? bufB : bufA;
            const int rounds = (op == 0 && !sq) ? nr : nr - 1;
            auto ld = [&](int, int, int p) -> T { return buf[p]; };
            auto st = [&](int, int, int p, T v) { buf[p] = v; };
            for (int r = 0; r < rounds; ++r) {
                run_round_rl<Ar, LayRow, RLOG, false, false>(sched_rl<RLOG>(log_n, r), log_n, 0,
                                                     sched_s0<RLOG>(log_n, r), pr.WCf, ar, false,
                                                     ld, st);
                __syncthreads();
            }
        }
        {
            // last forward round of B (or A), product, first inverse round
            const int r = nr - 1;
            const int rl = sched_rl<RLOG>(log_n, r), s0 = sched_s0<RLOG>(log_n, r);
            const int d_log = log_n - s0 - rl;
            const int nsub = 1 << (log_n - rl);
            const bool final_round = (nr == 1);
            T* src = sq ? bufA : bufB;
            for (int sp = threadIdx.x; sp < nsub; sp += NT) {
                const int j = sp & ((1 << d_log) - 1);
                const int g = sp >> d_log;
                const int base = (g << (d_log + rl)) + j;
                const int p0 = LayRow::p(base);   // last round: stride 1 (d_log = 0)
                T x[1 << RLOG];
#define BW_SMALL_FUSED(RL)                                                             \
    {                                                                                  \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) x[k] = src[p0 + k];     \
        ct_stages<Ar, RL, false>(x, s0, g, pr.WCf, ar, false);                         \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) {                        \
            const T xa = ar.fwd_to_2p(x[k]);                                           \
            const T ya = sq ? xa : ar.fwd_to_2p(bufA[p0 + k]);                         \
            x[k] = ar.mont(xa, ya);                                                    \
        }                                                                              \
        gs_stages<Ar, RL, false>(x, s0, g, pr.WCi, ar);                                \
        _Pragma("unroll") for (int k = 0; k < (1 << RL); ++k) {                        \
            if (final_round) st_res(base + k, x[k]); else bufA[p0 + k] = x[k];         \
        }                                                                              \
    }
                if (rl == RLOG) {
                    BW_SMALL_FUSED(RLOG)
                } else if (rl == 3) {
                    BW_SMALL_FUSED(3)
                } else if (rl == 2) {
                    BW_SMALL_FUSED(2)
                } else {
                    BW_SMALL_FUSED(1)
                }
#undef BW_SMALL_FUSED
            }
            __syncthreads();
        }
        for (int r = nr - 2; r >= 0; --r) {
            const bool last = (r == 0);
            auto st = [&](int, int idx, int p, T v) {
                if (last) {
                    st_res(idx, v);
                } else {
                    bufA[p] = v;
                }
            };
            run_round_rl<Ar, LayRow, RLOG, true, false>(sched_rl<RLOG>(log_n, r), log_n, 0,
                                                sched_s0<RLOG>(log_n, r), pr.WCi, ar, false, ldA,
                                                st);
            __syncthreads();
        }
    }

    // ---- Garner + carry, tile by tile; the carry into a tile is the previous
    // tile's last carry words (s_cin) plus its chain carry-out bit (s_eps)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const size_t NL = (size_t)n / CPW, M = (size_t)d.la + d.lb;
    const size_t words = NL > M ? NL : M;
    if (tid == 0) {
        s_cin[0] = s_cin[1] = s_cin[2] = 0;
        s_eps = 0;
    }
    __syncthreads();
    uint32_t bad = 0;
    for (size_t t0 = 0; t0 < words; t0 += (size_t)NT * E) {
        const size_t j0 = t0 + (size_t)tid * E;
        unsigned __int128 Dg[E];
        garner_digits<Ar, SPLIT16, E, false>(P, res, n, j0, NL, Dg, &bad);
        uint32_t l[E], X[3];
        {
            unsigned __int128 acc = 0;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                acc += Dg[e];
                l[e] = (uint32_t)acc;
                acc >>= 32;
            }
            X[0] = (uint32_t)acc;
            X[1] = (uint32_t)(acc >> 32);
            X[2] = (uint32_t)(acc >> 64);
        }
        uint32_t PX[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) PX[q] = __shfl_up_sync(0xffffffffu, X[q], 1);
        if (lane == 31) {
            s_lastx[warp][0] = X[0];
            s_lastx[warp][1] = X[1];
            s_lastx[warp][2] = X[2];
        }
        __syncthreads();
        if (lane == 0) {
#pragma unroll
            for (int q = 0; q < 3; ++q) PX[q] = warp > 0 ? s_lastx[warp - 1][q] : s_cin[q];
        }
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
        const uint32_t eps_in = s_eps;
        const uint32_t mc = chain_mine(cm, s_w, eps_in);
        const uint32_t cout = chain_out(s_w, eps_in);
        {
            uint64_t c = mc;
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const uint64_t s = (uint64_t)S[e] + c;
                if (j0 + e < M) d.out[j0 + e] = (uint32_t)s;
                c = s >> 32;
            }
        }
        __syncthreads();  // every thread has read s_cin, s_eps, s_lastx, s_w
        if (tid == NT - 1) {
            s_cin[0] = X[0];
            s_cin[1] = X[1];
            s_cin[2] = X[2];
        }
        if (tid == 0) s_eps = cout;
        __syncthreads();
    }
    if (bad) atomicOr(err, 2u);
}

template <class Ar, bool SPLIT16, int NT>
__global__ void __launch_bounds__(NT, ks_min_blocks<Ar>(NT))
ks_product(const PlanDev<Ar> P, const BatchProd* __restrict__ D, typename Ar::T* scratch,
           uint32_t* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ks_product_body<Ar, SPLIT16, NT>(P, D[blockIdx.x], scratch, err, smem_raw);
}

// Persistent form of the small buckets of one prime path
// (BW_BATCH_PERSISTENT): a grid of a few CTAs per SM pulls work items --
// (bucket, product) pairs, largest transforms first -- from a device queue
// (an atomic head) and runs each as ks_product does, reading the bucket's
// plan and descriptor from device arrays.  The queue head is cleared before
// every run; a CTA stops at the first item past the end.  No waits.
struct SmallItem {
    uint32_t bucket;
    uint32_t prod;
};
template <class Ar>
struct SmallBucketDev {
    PlanDev<Ar> plan;
    const BatchProd* desc;
    typename Ar::T* scratch;
};
template <class Ar, bool SPLIT16, int NT>
__global__ void __launch_bounds__(NT, ks_min_blocks<Ar>(NT))
kq_small(const SmallBucketDev<Ar>* __restrict__ buckets, const SmallItem* __restrict__ items,
         uint32_t count, uint32_t* __restrict__ head, uint32_t* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(head, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= count) break;
        const SmallItem w = items[it];
        const SmallBucketDev<Ar>& b = buckets[w.bucket];
        ks_product_body<Ar, SPLIT16, NT>(b.plan, b.desc[w.prod], b.scratch, err, smem_raw);
        __syncthreads();  // every thread has read s_item and left the body
    }
}

}  // namespace bw
