// crt.h -- host CRT helpers, compatible with nikitaborisov/birdwing
// include/crt.h:1-30 (implemented in birdwing_b200/csrc/compat/crt.cpp).
#pragma once
#include <cstdint>
#include <vector>

#include "crt_utils.h"

using namespace std;

// two-modulus CRT parameters
struct CRT2Params {
    TestDataTypeUint p1;
    TestDataTypeUint p2;
    TestDataTypeUint p1_inv_mod_p2;
    unsigned __int128 modulus;

    CRT2Params(TestDataTypeUint _p1, TestDataTypeUint _p2);
};

// x mod p1*p2 from (x mod p1, x mod p2)
unsigned __int128 crt_combine_2(const CRT2Params& params, TestDataTypeUint a_mod_p1,
                                TestDataTypeUint b_mod_p2);

// x mod prod(primes) from residues (value kept mod 2^128)
unsigned __int128 crt_combine_many(const vector<TestDataTypeUint>& primes,
                                   const vector<TestDataTypeUint>& residues);
