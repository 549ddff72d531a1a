// crt_utils.h -- host helpers, compatible with nikitaborisov/birdwing
// include/crt_utils.h (implemented in birdwing_b200/csrc/compat/crt.cpp).
#pragma once
#include <cstdint>

#include "config.h"

using namespace std;

// decimal print of an unsigned 128-bit value
void print_u128(unsigned __int128 x);

// a^-1 mod m (a, m coprime, m < 2^63)
uint64_t modinv_u64(uint64_t a, uint64_t m);
