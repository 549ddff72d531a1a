// bw_arith.cuh -- exact modular arithmetic for the two prime paths.
//
// Residues are kept lazily reduced (Harvey): the forward Cooley-Tukey
// butterfly keeps values in [0, 4p), the inverse Gentleman-Sande butterfly in
// [0, 2p).  Both need 4p < 2^bits, which is why the 32-bit path uses primes
// below 2^30 and the 64-bit path primes below 2^62.
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

    __device__ __forceinline__ T red2(T a) const { return a >= p2 ? a - p2 : a; }
    __device__ __forceinline__ T red1(T a) const { return a >= p ? a - p : a; }
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
};

struct Ar64 {
    using T = uint64_t;
    static constexpr int BITS = 64;
    uint64_t p;
    uint64_t p2;    // 2p
    uint64_t pinv;  // -p^-1 mod 2^64

    __device__ __forceinline__ T red2(T a) const { return a >= p2 ? a - p2 : a; }
    __device__ __forceinline__ T red1(T a) const { return a >= p ? a - p : a; }
    __device__ __forceinline__ T shoup(T x, T w, T wq) const {
        const uint64_t q = __umul64hi(x, wq);
        return x * w - q * p;
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
    __device__ __forceinline__ void ct(T& a, T& b, T w, T wq) const {
        const T x = red2(a);
        const T t = shoup(b, w, wq);
        a = x + t;
        b = x - t + p2;
    }
    __device__ __forceinline__ void gs(T& a, T& b, T w, T wq) const {
        const T u = a + b;
        const T v = a - b + p2;
        a = red2(u);
        b = shoup(v, w, wq);
    }
};

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
