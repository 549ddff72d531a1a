// ntt_limits.h -- size admission, compatible with nikitaborisov/birdwing
// include/ntt_limits.h:9-31.  The functions are pure functions of the
// `moduli` / `roots_of_unity_max` tables of config.h (implemented in
// birdwing_b200/csrc/compat/ntt_limits.cpp).  libbirdwing's own admission is
// bw_size_supported / bw_limits (birdwing.h).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "config.h"

int max_logN_for_prime(uint64_t p);                        // v2(p - 1)
int max_root_logN(TestDataTypeUint root, TestDataTypeUint p);  // log2 order of root
int max_supported_logN();
size_t max_supported_N();

// largest square operand length L for which both the NTT and CRT bounds hold
size_t max_supported_limb_count();

size_t padded_ntt_size(size_t L_A, size_t L_B);

bool ntt_size_supported(size_t N, std::string* why = nullptr);

// min(L_A, L_B) * (2^INPUT_LIMB_BITS - 1)^2 < product(moduli)
bool crt_coefficient_bound_satisfied(size_t L_A, size_t L_B, std::string* why = nullptr);

bool multiply_size_supported(size_t L_A, size_t L_B, std::string* why = nullptr);

// print the reason to stderr and exit(1) when unsupported (source
// compatibility with the reference; the C ABI returns BW_ESIZE instead)
void ensure_ntt_size_supported(size_t N);
void ensure_multiply_size_supported(size_t L_A, size_t L_B);
