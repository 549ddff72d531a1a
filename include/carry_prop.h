// carry_prop.h -- segmented carry propagation kernels, compatible with
// nikitaborisov/birdwing include/carry_prop.h:7-49 (same signatures; they are
// launched by callers as <<<num_segs, 1>>> with a host loop that re-runs the
// fixup while *escape_flag is set).  Implemented in
// birdwing_b200/csrc/compat/carry_prop.cu.  libbirdwing's own pipeline uses a
// single decoupled-look-back kernel instead.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "config.h"

__global__ void carry_intra_segment_kernel(const uint64_t* __restrict__ C_hi,
                                           const uint64_t* __restrict__ C_lo,
                                           OutputLimbType* __restrict__ out,
                                           int64_t* __restrict__ seg_carry, size_t N);

__global__ void carry_inter_segment_kernel(int64_t* __restrict__ seg_carry, size_t num_segs);

__global__ void carry_fixup_kernel(OutputLimbType* __restrict__ out,
                                   int64_t* __restrict__ seg_carry, size_t N, size_t num_segs,
                                   int* __restrict__ escape_flag);

#if defined(NATIVE_HOST_LIMBS)
__global__ void carry_intra_segment_kernel_u160(const uint64_t* __restrict__ C_lo,
                                                const uint64_t* __restrict__ C_mid,
                                                const uint32_t* __restrict__ C_hi,
                                                OutputLimbType* __restrict__ out,
                                                uint64_t* __restrict__ seg_carry_lo,
                                                uint64_t* __restrict__ seg_carry_mid,
                                                uint32_t* __restrict__ seg_carry_hi, size_t N);

__global__ void carry_inter_segment_kernel_u160(uint64_t* __restrict__ seg_carry_lo,
                                                uint64_t* __restrict__ seg_carry_mid,
                                                uint32_t* __restrict__ seg_carry_hi,
                                                size_t num_segs);

__global__ void carry_fixup_kernel_u160(OutputLimbType* __restrict__ out,
                                        uint64_t* __restrict__ seg_carry_lo,
                                        uint64_t* __restrict__ seg_carry_mid,
                                        uint32_t* __restrict__ seg_carry_hi, size_t N,
                                        size_t num_segs, int* __restrict__ escape_flag);
#endif
