// multiply.h -- one-shot product, compatible with nikitaborisov/birdwing
// include/multiply.h:9-23.  Implemented over the C ABI (bw_multiply_host_once)
// in birdwing_b200/csrc/compat/host_multiply.cpp.
#pragma once
#include <chrono>
#include <cstdint>
#include <vector>

#include "config.h"

using limb_t = OutputLimbType;

#if !defined(NATIVE_HOST_LIMBS)
// C = A * B with u32 limbs; C gets A.size() + B.size() limbs
void host_multiply_merge(const vector<uint32_t>& A, const vector<uint32_t>& B,
                         vector<OutputLimbType>& C, chrono::duration<double, milli>& duration);
#endif

#if defined(NATIVE_HOST_LIMBS)
// C = A * B with u64 limbs
void host_multiply_merge_native(const vector<uint64_t>& A, const vector<uint64_t>& B,
                                vector<uint64_t>& C, chrono::duration<double, milli>& duration);
#endif
