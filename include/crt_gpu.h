// crt_gpu.h -- Garner CRT on the GPU, compatible with
// nikitaborisov/birdwing include/crt_gpu.h:11-41 (implemented in
// birdwing_b200/csrc/compat/crt_gpu.cu).  The product pipeline of
// libbirdwing fuses Garner into its carry kernel; these entry points keep the
// reference's stage-level API for callers that use it directly.
#pragma once

#include <vector>

#include "config.h"
#include "crt_utils.h"

using namespace std;

// Garner constants of NUM_MODULI primes (host side, uploaded to constant
// memory by upload_garner_params).
struct CRTGarnerParams {
    uint64_t primes[NUM_MODULI];
    uint64_t inv[NUM_MODULI];       // inv[i] = (p0 ... p_{i-1})^-1 mod p_i
    uint64_t prefix_M[NUM_MODULI];  // prefix_M[i] = (p0 ... p_{i-1}) mod p_i
    uint64_t M_mod_table[NUM_MODULI][NUM_MODULI];  // [k][i] = (p0..p_{k-1}) mod p_i
    uint64_t barrett_m[NUM_MODULI];  // floor(2^64 / p_i) (32-bit residues)
};

CRTGarnerParams compute_garner_params(const vector<TestDataTypeUint>& primes);

void upload_garner_params(const CRTGarnerParams& params);

// device pointers of the NUM_MODULI residue arrays crt_combine_gpu reads
void upload_residue_ptrs(const vector<TestDataTypeUint*>& c_dev);

// x_i = CRT of the residues at index i, as (C_hi[i] << 64) | C_lo[i]
void crt_combine_gpu(uint64_t* d_C_hi, uint64_t* d_C_lo, int N);

#if defined(NATIVE_HOST_LIMBS)
// x_i = C_lo[i] | C_mid[i] << 64 | C_hi[i] << 128
void crt_combine_gpu_u160(uint64_t* d_C_lo, uint64_t* d_C_mid, uint32_t* d_C_hi, int N);
#endif
