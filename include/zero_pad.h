// zero_pad.h -- limb widening / reduction with zero padding, compatible with
// nikitaborisov/birdwing include/zero_pad.h:6-21 (implemented in
// birdwing_b200/csrc/compat/zero_pad.cu).  libbirdwing's pipeline pads
// virtually inside its first transform pass instead.
#pragma once

#include <cuda_runtime.h>

#include "config.h"

// d_dst[i] = i < L ? d_src[i] : 0 for i < N
void zero_pad_gpu(const uint32_t* d_src, TestDataTypeUint* d_dst, size_t L, size_t N,
                  cudaStream_t stream);

#if defined(NATIVE_HOST_LIMBS)
// d_dst[i] = i < L ? d_src[i] mod modulus : 0 for i < N
void zero_pad_gpu_u64(const uint64_t* d_src, TestDataTypeUint* d_dst, size_t L, size_t N,
                      TestDataTypeUint modulus, cudaStream_t stream);
#endif
