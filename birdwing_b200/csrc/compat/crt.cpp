// crt.cpp -- host CRT helpers.  Reference: src/crt.cpp:6-86 and
// src/crt_utils.cpp:9-50 (same functions and semantics).
#include "crt.h"

#include <cassert>
#include <cstdio>

void print_u128(unsigned __int128 x) {
    char buf[48];
    int i = 47;
    buf[i] = '\0';
    do {
        buf[--i] = (char)('0' + (int)(x % 10));
        x /= 10;
    } while (x != 0);
    std::printf("%s", buf + i);
}

uint64_t modinv_u64(uint64_t a, uint64_t m) {
    // extended Euclid on signed 128-bit values (no overflow for m < 2^64)
    __int128 r0 = m, r1 = a % m, t0 = 0, t1 = 1;
    while (r1 != 0) {
        const __int128 q = r0 / r1;
        const __int128 r2 = r0 - q * r1;
        r0 = r1;
        r1 = r2;
        const __int128 t2 = t0 - q * t1;
        t0 = t1;
        t1 = t2;
    }
    assert(r0 == 1);
    if (t0 < 0) t0 += m;
    return (uint64_t)t0;
}

CRT2Params::CRT2Params(TestDataTypeUint _p1, TestDataTypeUint _p2) : p1(_p1), p2(_p2) {
    modulus = (unsigned __int128)p1 * p2;
    p1_inv_mod_p2 = (TestDataTypeUint)modinv_u64(p1 % p2, p2);
}

unsigned __int128 crt_combine_2(const CRT2Params& params, TestDataTypeUint a_mod_p1,
                                TestDataTypeUint b_mod_p2) {
    const uint64_t p2 = params.p2;
    const uint64_t a2 = (uint64_t)a_mod_p1 % p2;
    const uint64_t d = b_mod_p2 >= a2 ? b_mod_p2 - a2 : b_mod_p2 + p2 - a2;
    const uint64_t t = (uint64_t)((unsigned __int128)d * params.p1_inv_mod_p2 % p2);
    return (unsigned __int128)a_mod_p1 + (unsigned __int128)params.p1 * t;
}

unsigned __int128 crt_combine_many(const vector<TestDataTypeUint>& primes,
                                   const vector<TestDataTypeUint>& residues) {
    assert(primes.size() == residues.size() && !primes.empty());
    unsigned __int128 x = 0, M = 1;
    for (size_t i = 0; i < primes.size(); ++i) {
        const uint64_t p = primes[i];
        const uint64_t xm = (uint64_t)(x % p);
        const uint64_t r = residues[i] % p;
        const uint64_t d = r >= xm ? r - xm : r + p - xm;
        const uint64_t k = (uint64_t)((unsigned __int128)d * modinv_u64((uint64_t)(M % p), p) % p);
        x += M * k;
        M *= p;
    }
    return x;
}
