// ntt_limits.cpp -- size admission as pure functions of the `moduli` and
// `roots_of_unity_max` tables.  Reference rules: src/ntt_limits.cpp:14-280
// (NTT length <= min over primes of min(v2(p-1), log2 root order); padded
// length next_pow2(L_A + L_B - 1); CRT bound min(L_A, L_B) (2^b - 1)^2 <
// prod(p), in long double when input limbs are 64-bit).
#include "ntt_limits.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <limits>

using namespace std;

namespace {

uint64_t sqmod(uint64_t r, uint64_t p) { return (uint64_t)((unsigned __int128)r * r % p); }

int log_limit(size_t i) {
    return min(max_logN_for_prime(moduli[i]), max_root_logN(roots_of_unity_max[i], moduli[i]));
}

bool wide_inputs() { return INPUT_LIMB_BITS == 64; }

unsigned __int128 prod_u128() {
    unsigned __int128 m = 1;
    for (int i = 0; i < NUM_MODULI; ++i) m *= (unsigned __int128)moduli[i];
    return m;
}

long double prod_ld() {
    long double m = 1.0L;
    for (int i = 0; i < NUM_MODULI; ++i) m *= (long double)moduli[i];
    return m;
}

long double limb_max_ld() {
    return wide_inputs() ? (long double)UINT64_MAX : (long double)OUTPUT_LIMB_MASK;
}

size_t crt_limb_limit() {
    if (wide_inputs()) {
        const long double q = prod_ld() / ((long double)UINT64_MAX * (long double)UINT64_MAX);
        return q > (long double)numeric_limits<size_t>::max() ? numeric_limits<size_t>::max()
                                                              : (size_t)q;
    }
    const unsigned __int128 sq = (unsigned __int128)OUTPUT_LIMB_MASK * OUTPUT_LIMB_MASK;
    const unsigned __int128 q = (prod_u128() - 1) / sq;
    return q > numeric_limits<size_t>::max() ? numeric_limits<size_t>::max() : (size_t)q;
}

bool logn_ok(int logN, string* why) {
    for (int i = 0; i < NUM_MODULI; ++i) {
        const int lim = log_limit(i);
        if (logN > lim) {
            if (why)
                *why = "NTT size N=2^" + to_string(logN) + " exceeds modulus " + to_string(i) +
                       " (p=" + to_string((uint64_t)moduli[i]) + ", max 2^" + to_string(lim) +
                       ")";
            return false;
        }
    }
    return true;
}

}  // namespace

int max_logN_for_prime(uint64_t p) {
    uint64_t x = p - 1;
    int k = 0;
    while (x && (x & 1) == 0) {
        x >>= 1;
        ++k;
    }
    return k;
}

int max_root_logN(TestDataTypeUint root, TestDataTypeUint p) {
    uint64_t r = (uint64_t)root % p;
    if (r == 0) return 0;
    for (int k = 0; k < 62; ++k) {
        if (r == 1) return k;
        r = sqmod(r, p);
    }
    return 62;
}

int max_supported_logN() {
    int m = numeric_limits<int>::max();
    for (int i = 0; i < NUM_MODULI; ++i) m = min(m, log_limit(i));
    return m;
}

size_t max_supported_N() {
    const int l = max_supported_logN();
    return l < 0 ? 0 : (size_t)1 << l;
}

size_t padded_ntt_size(size_t L_A, size_t L_B) {
    const size_t need = L_A + L_B - 1;
    size_t n = 1;
    while (n < need) n <<= 1;
    return n;
}

size_t max_supported_limb_count() {
    const int l = max_supported_logN();
    if (l <= 0) return 0;
    return min((size_t)1 << (l - 1), crt_limb_limit());
}

bool crt_coefficient_bound_satisfied(size_t L_A, size_t L_B, string* why) {
    if (L_A == 0 || L_B == 0) {
        if (why) *why = "operand limb count must be positive";
        return false;
    }
    const size_t terms = min(L_A, L_B);
    bool ok;
    if (wide_inputs()) {
        const long double lm = limb_max_ld();
        ok = (long double)terms * lm * lm < prod_ld();
    } else {
        const unsigned __int128 sq = (unsigned __int128)OUTPUT_LIMB_MASK * OUTPUT_LIMB_MASK;
        ok = (unsigned __int128)terms * sq < prod_u128();
    }
    if (!ok && why)
        *why = "max convolution coefficient for L_A=" + to_string(L_A) + ", L_B=" + to_string(L_B) +
               " (terms=" + to_string(terms) + ", limb=" + to_string(INPUT_LIMB_BITS) +
               "-bit) exceeds CRT modulus product";
    return ok;
}

bool ntt_size_supported(size_t N, string* why) {
    if (N == 0) {
        if (why) *why = "NTT size N must be positive";
        return false;
    }
    if (N & (N - 1)) {
        if (why) *why = "NTT size N=" + to_string(N) + " is not a power of two";
        return false;
    }
    int logN = 0;
    while (((size_t)1 << logN) < N) ++logN;
    return logn_ok(logN, why);
}

bool multiply_size_supported(size_t L_A, size_t L_B, string* why) {
    if (L_A == 0 || L_B == 0) {
        if (why) *why = "operand limb count must be positive";
        return false;
    }
    if (!ntt_size_supported(padded_ntt_size(L_A, L_B), why)) return false;
    return crt_coefficient_bound_satisfied(L_A, L_B, why);
}

void ensure_ntt_size_supported(size_t N) {
    string why;
    if (ntt_size_supported(N, &why)) return;
    cerr << "[NTT] Unsupported size: " << why << "\n"
         << "[NTT] Max supported N=2^" << max_supported_logN() << " (" << max_supported_N()
         << "), max L=2^" << (max_supported_logN() - 1) << " (" << max_supported_limb_count()
         << ")\n";
    exit(1);
}

void ensure_multiply_size_supported(size_t L_A, size_t L_B) {
    string why;
    if (multiply_size_supported(L_A, L_B, &why)) return;
    cerr << "[NTT] Unsupported multiply: " << why << "\n"
         << "[NTT] Max supported N=2^" << max_supported_logN() << " (" << max_supported_N()
         << "), max L (square)=2^" << (max_supported_logN() - 1) << " ("
         << max_supported_limb_count() << "), max L (CRT only)=" << crt_limb_limit() << "\n";
    exit(1);
}
