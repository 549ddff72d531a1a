// bw_arith.cuh -- exact modular arithmetic for the two prime paths.
//
// Residues are kept lazily reduced (Harvey).  On the 32-bit path the forward
// Cooley-Tukey butterfly keeps values in [0, 4p) and the inverse
// Gentleman-Sande butterfly in [0, 2p), which needs 4p < 2^32 (primes below
// 2^30).  The 64-bit path's primes are below 2^58, which leaves its forward
// transform 64x headroom (see Ar64).
//
// Multiplication by a precomputed constant w uses Shoup's method with the
// companion wq = floor(w * 2^bits / p): q = hi(x * wq), r = x*w - q*p lies in
// [0, 2p) for every x < 2^bits.  Products of two variables (the pointwise
// step) use Montgomery multiplication; its 2^-bits factor is cancelled by a
// 2^bits folded into the inverse transform's scale constant.
//
// The reference computes these products with a plain `%` on 64/128-bit
// values (pointwise_mul_kernel, src/gpu_ntt.cu:216-238; mulmod64,
// src/crt_gpu.cu:47-67), which is a software division on the GPU.
#pragma once
#include <cstdint>

namespace bw {

template <typename T>
struct alignas(2 * sizeof(T)) Tw {
    T w;
    T wq;
};

struct Ar32 {
    using T = uint32_t;
    static constexpr int BITS = 32;
    uint32_t p;
    uint32_t p2;    // 2p
    uint32_t pinv;  // -p^-1 mod 2^32
    uint32_t r32;   // 2^32 mod p
    uint32_t r32q;  // Shoup companion of r32
    uint32_t oneq;  // floor(2^32 / p): Shoup companion of 1
    double pinv_d;  // 2^32 / p, for companions of twiddles built on the device

    __device__ __forceinline__ T red2(T a) const { return min(a, a - p2); }
    __device__ __forceinline__ T red1(T a) const { return min(a, a - p); }
    // x < 2^32, w < p: returns x*w mod p in [0, 2p)
    __device__ __forceinline__ T shoup(T x, T w, T wq) const {
        const uint32_t q = __umulhi(x, wq);
        return x * w - q * p;
    }
    // a, b < 2p: returns a*b*2^-32 mod p in [0, 2p)
    __device__ __forceinline__ T mont(T a, T b) const {
        const uint64_t t = (uint64_t)a * b;
        const uint32_t m = (uint32_t)t * pinv;
        return (uint32_t)((t + (uint64_t)m * p) >> 32);
    }
    // forward CT butterfly, inputs/outputs in [0, 4p)
    __device__ __forceinline__ void ct(T& a, T& b, T w, T wq) const {
        const T x = red2(a);
        const T t = shoup(b, w, wq);
        a = x + t;
        b = x - t + p2;
    }
    // inverse GS butterfly, inputs/outputs in [0, 2p)
    __device__ __forceinline__ void gs(T& a, T& b, T w, T wq) const {
        const T u = a + b;
        const T v = a - b + p2;
        a = red2(u);
        b = shoup(v, w, wq);
    }
    // twiddle-1 butterflies of stage 0 (inputs known to be in [0, 2p))
    __device__ __forceinline__ void ct1(T& a, T& b) const {
        const T x = a;
        a = x + b;
        b = x - b + p2;
    }
    __device__ __forceinline__ void gs1(T& a, T& b) const {
        const T x = a;
        a = red2(x + b);
        b = red2(x - b + p2);
    }
    // forward-transform output range [0, 4p) -> [0, 2p)
    __device__ __forceinline__ T fwd_to_2p(T a) const { return red2(a); }
    // inverse-transform output range [0, 2p) -> [0, p)
    __device__ __forceinline__ T inv_out(T a) const { return red1(a); }
    // x * w for a twiddle applied between transform passes, in [0, 2p)
    __device__ __forceinline__ T mulc(T x, T w, T wq) const { return shoup(x, w, wq); }
    // Shoup companion floor(w 2^32 / p) of w < p: a double-precision estimate
    // w (2^32 / p) is within 2^-20 of the quotient (below 2^32, relative error
    // under 2^-51), so its floor is exact or one off, and the exact remainder
    // w 2^32 - q p (in [-p, 2p)) decides the correction
    __device__ __forceinline__ T companion(T w) const {
        uint32_t q = (uint32_t)((double)w * pinv_d);
        const int64_t r = (int64_t)((((uint64_t)w) << 32) - (uint64_t)q * p);
        if (r < 0) {
            --q;
        } else if (r >= (int64_t)p) {
            ++q;
        }
        return q;
    }
    // a 64-bit coefficient x = h 2^32 + l reduced to [0, 2p): h (2^32 mod p)
    // and l * 1 by Shoup, each in [0, 2p), their sum below 4p
    __device__ __forceinline__ T reduce64(uint64_t x) const {
        const T h = shoup((uint32_t)(x >> 32), r32, r32q);
        const T l = shoup((uint32_t)x, 1u, oneq);
        return red2(h + l);
    }
};

// The 64-bit path's primes are p = c 2^32 + 1 below 2^58, so 64p < 2^64.
// Every multiplication by a constant inside and between the transforms uses
// the truncated Shoup quotient, which omits the x0*v0 partial product (q may
// be 2 short, so the product lies in [0, 3p)).  The forward (CT) butterfly
// adds without reducing: from inputs below 3p its stage-0 sums stay below 6p
// and every later stage adds less than 3p, so s stages stay below 3p (s + 1)
// -- below 64p for the at most 13 stages one pass runs (the headroom the
// 58-bit primes buy: with primes near 2^62 every butterfly reduced its input).
// The inverse (GS) transform keeps values in [0, 3p): sums are reduced by one
// conditional subtraction of 3p, differences are offset by 3p (6p < 2^64).
// A forward output enters the pointwise product reduced to [0, 2p) by an
// exact Shoup multiplication by 1.  Garner and the final scalings use the
// exact quotient.
struct Ar64 {
    using T = uint64_t;
    static constexpr int BITS = 64;
    uint64_t p;
    uint64_t p2;    // 2p
    uint64_t pinv;  // -p^-1 mod 2^64
    uint32_t c;     // p = c * 2^32 + 1
    uint32_t c3;    // 3c
    uint64_t p3;    // 3p
    uint64_t p4;    // 4p
    uint64_t mu_lo; // floor(2^128 / p) = mu_hi 2^64 + mu_lo
    uint32_t mu_hi;
    uint64_t oneq;  // floor(2^64 / p): Shoup companion of 1

    __device__ __forceinline__ T red2(T a) const { return min(a, a - p2); }
    __device__ __forceinline__ T red1(T a) const { return min(a, a - p); }
    // x < 2^64, w < p: x*w mod p in [0, 2p).  The quotient q = hi64(x * wq)
    // is exact and built from 32x32->64 multiply-adds (mad.wide.u32) whose
    // 64-bit addends never overflow:
    //   T = x0 v1 + hi(x0 v0),  W = x1 v0 + lo(T),  q = x1 v1 + hi(W) + hi(T).
    // Because p = c 2^32 + 1, q*p mod 2^64 = q + (q0 c) 2^32 costs one
    // multiply-add; r = lo64(x w) - lo64(q p).
    __device__ __forceinline__ T shoup(T x, T w, T wq) const {
        uint64_t r;
        asm("{\n\t"
            ".reg .u32 x0, x1, v0, v1, w0, w1, h, t0, t1, s0, s1, f0, f1, q0, q1, l0, l1, qh, r0, r1;\n\t"
            ".reg .u64 A, TT, WW, F, Q, L;\n\t"
            "mov.b64 {x0, x1}, %1;\n\t"
            "mov.b64 {w0, w1}, %2;\n\t"
            "mov.b64 {v0, v1}, %3;\n\t"
            "mul.hi.u32 h, x0, v0;\n\t"
            "mov.b64 A, {h, 0};\n\t"
            "mad.wide.u32 TT, x0, v1, A;\n\t"
            "mov.b64 {t0, t1}, TT;\n\t"
            "mov.b64 A, {t0, 0};\n\t"
            "mad.wide.u32 WW, x1, v0, A;\n\t"
            "mov.b64 {s0, s1}, WW;\n\t"
            "add.cc.u32 f0, s1, t1;\n\t"
            "addc.u32 f1, 0, 0;\n\t"
            "mov.b64 F, {f0, f1};\n\t"
            "mad.wide.u32 Q, x1, v1, F;\n\t"
            "mov.b64 {q0, q1}, Q;\n\t"
            "mul.wide.u32 L, x0, w0;\n\t"
            "mov.b64 {l0, l1}, L;\n\t"
            "mad.lo.u32 l1, x0, w1, l1;\n\t"
            "mad.lo.u32 l1, x1, w0, l1;\n\t"
            "mad.lo.u32 qh, q0, %4, q1;\n\t"
            "sub.cc.u32 r0, l0, q0;\n\t"
            "subc.u32 r1, l1, qh;\n\t"
            "mov.b64 %0, {r0, r1};\n\t"
            "}"
            : "=l"(r)
            : "l"(x), "l"(w), "l"(wq), "r"(c));
        return r;
    }
    // a, b < 2p: returns a*b*2^-64 mod p in [0, 2p).  The low word of
    // t + m*p is zero by construction, so its carry is (lo != 0).
    __device__ __forceinline__ T mont(T a, T b) const {
        const uint64_t lo = a * b;
        const uint64_t hi = __umul64hi(a, b);
        const uint64_t m = lo * pinv;
        const uint64_t mh = __umul64hi(m, p);
        return hi + mh + (lo != 0 ? 1ull : 0ull);
    }
    // x < 2^64, w < p: x*w mod p in [0, 3p) from the truncated quotient
    // q' = x1 v1 + hi(x0 v1 + x1 v0) (the dropped x0 v0 term and the dropped
    // low bits make q' at most 2 below hi64(x * wq)).
    __device__ __forceinline__ T shoup3(T x, T w, T wq) const {
        uint64_t r;
        asm("{\n\t"
            ".reg .u32 x0, x1, v0, v1, w0, w1, t0, t1, s0, s1, f0, f1, q0, q1, l0, l1, qh, r0, r1;\n\t"
            ".reg .u64 A, TT, WW, F, Q, L;\n\t"
            "mov.b64 {x0, x1}, %1;\n\t"
            "mov.b64 {w0, w1}, %2;\n\t"
            "mov.b64 {v0, v1}, %3;\n\t"
            "mul.wide.u32 TT, x0, v1;\n\t"
            "mov.b64 {t0, t1}, TT;\n\t"
            "mov.b64 A, {t0, 0};\n\t"
            "mad.wide.u32 WW, x1, v0, A;\n\t"
            "mov.b64 {s0, s1}, WW;\n\t"
            "add.cc.u32 f0, s1, t1;\n\t"
            "addc.u32 f1, 0, 0;\n\t"
            "mov.b64 F, {f0, f1};\n\t"
            "mad.wide.u32 Q, x1, v1, F;\n\t"
            "mov.b64 {q0, q1}, Q;\n\t"
            "mul.wide.u32 L, x0, w0;\n\t"
            "mov.b64 {l0, l1}, L;\n\t"
            "mad.lo.u32 l1, x0, w1, l1;\n\t"
            "mad.lo.u32 l1, x1, w0, l1;\n\t"
            "mad.lo.u32 qh, q0, %4, q1;\n\t"
            "sub.cc.u32 r0, l0, q0;\n\t"
            "subc.u32 r1, l1, qh;\n\t"
            "mov.b64 %0, {r0, r1};\n\t"
            "}"
            : "=l"(r)
            : "l"(x), "l"(w), "l"(wq), "r"(c));
        return r;
    }
    // forward CT butterfly: a + t and a - t + 3p with t = b w in [0, 3p), no
    // reduction (each stage grows the bound by less than 3p)
    __device__ __forceinline__ void ct(T& a, T& b, T w, T wq) const {
        const T x = a;
        const T t = shoup3(b, w, wq);  // [0, 3p)
        a = x + t;
        b = x - t + p3;
    }
    // inverse GS butterfly, inputs/outputs in [0, 3p)
    __device__ __forceinline__ void gs(T& a, T& b, T w, T wq) const {
        const T u = a + b;       // [0, 6p)
        const T v = a - b + p3;  // (0, 6p)
        a = min(u, u - p3);
        b = shoup3(v, w, wq);
    }
    // twiddle-1 butterflies of stage 0 (inputs in [0, 3p))
    __device__ __forceinline__ void ct1(T& a, T& b) const {
        const T x = a;
        a = x + b;
        b = x - b + p3;
    }
    __device__ __forceinline__ void gs1(T& a, T& b) const {
        const T u = a + b, v = a - b + p3;
        a = min(u, u - p3);
        b = min(v, v - p3);
    }
    // forward-transform output (any value below 2^64) -> [0, 2p)
    __device__ __forceinline__ T fwd_to_2p(T a) const { return shoup(a, 1, oneq); }
    // a 64-bit coefficient -> [0, 2p): the path's primes are c 2^32 + 1 with
    // 2^25 < c < 2^26, so q = x >> 58 is floor(x / p) or one less (x / p - q
    // < 1 + 2^-13), and x - q p = (x - q) - (q c) 2^32
    __device__ __forceinline__ T reduce_in(T x) const {
        const uint32_t q = (uint32_t)(x >> 58);
        return x - q - ((uint64_t)(q * c) << 32);
    }
    // inverse-transform output range [0, 3p) -> [0, p)
    __device__ __forceinline__ T inv_out(T a) const { return red1(min(a, a - p2)); }
    // x * w for a twiddle applied between transform passes, in [0, 3p)
    __device__ __forceinline__ T mulc(T x, T w, T wq) const { return shoup3(x, w, wq); }
    // Shoup companion floor(w 2^64 / p) of w < p by a Barrett step with
    // mu = floor(2^128 / p): the estimate is at most 2 short.
    __device__ __forceinline__ T companion(T w) const {
        uint64_t q = w * (uint64_t)mu_hi + __umul64hi(w, mu_lo);
        uint64_t r = 0 - q * p;
        if (r >= p) {
            ++q;
            r -= p;
        }
        if (r >= p) ++q;
        return q;
    }
};

// Twiddle load from shared memory (generic pointer into the CTA's tables).
template <typename T>
__device__ __forceinline__ Tw<T> ld_tw_s(const Tw<T>* p) {
    return *p;
}

template <typename T>
__device__ __forceinline__ Tw<T> ld_tw(const Tw<T>* p) {
    Tw<T> r;
    if constexpr (sizeof(T) == 8) {
        const ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
        r.w = v.x;
        r.wq = v.y;
    } else {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
        r.w = v.x;
        r.wq = v.y;
    }
    return r;
}

}  // namespace bw
