// wide_int.h -- 160-bit unsigned helper type of the native-limb CRT,
// compatible with nikitaborisov/birdwing include/wide_int.h:6-46.
#pragma once

#include <cstdint>

// value = lo + mid * 2^64 + hi * 2^128
struct U160 {
    uint64_t lo;
    uint64_t mid;
    uint32_t hi;
};

inline uint64_t u160_to_u64_lo(const U160& x) { return x.lo; }
inline uint64_t u160_to_u64_mid(const U160& x) { return x.mid; }
inline uint32_t u160_to_u32_hi(const U160& x) { return x.hi; }

inline bool u160_eq(const U160& a, const U160& b) {
    return a.lo == b.lo && a.mid == b.mid && a.hi == b.hi;
}

inline void u160_from_u128(uint64_t lo, uint64_t hi, U160& out) {
    out.lo = lo;
    out.mid = hi;
    out.hi = 0;
}

// a += b (mod 2^160)
inline void add160_host(U160& a, uint64_t b_lo, uint64_t b_mid, uint32_t b_hi) {
    const unsigned __int128 s0 = (unsigned __int128)a.lo + b_lo;
    const unsigned __int128 s1 = (unsigned __int128)a.mid + b_mid + (uint64_t)(s0 >> 64);
    a.lo = (uint64_t)s0;
    a.mid = (uint64_t)s1;
    a.hi = a.hi + b_hi + (uint32_t)(s1 >> 64);
}

// (M_hi:M_lo) * k as a 160-bit (lo, mid, hi) triple (the top bits beyond 160
// are dropped)
inline void mul128x64_host(uint64_t M_hi, uint64_t M_lo, uint64_t k, uint64_t& out_lo,
                           uint64_t& out_mid, uint32_t& out_hi) {
    const unsigned __int128 lo = (unsigned __int128)M_lo * k;
    const unsigned __int128 hi = (unsigned __int128)M_hi * k + (uint64_t)(lo >> 64);
    out_lo = (uint64_t)lo;
    out_mid = (uint64_t)hi;
    out_hi = (uint32_t)(hi >> 64);
}
