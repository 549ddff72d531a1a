// zero_pad.cu -- widen (or reduce) limbs into a zero-padded residue buffer.
// Reference: src/zero_pad.cu:3-57 (same interface; grid-stride launch).
#include "zero_pad.h"

namespace {
__global__ void pad_u32(const uint32_t* __restrict__ src, TestDataTypeUint* __restrict__ dst,
                        size_t L, size_t N) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = i < L ? (TestDataTypeUint)src[i] : (TestDataTypeUint)0;
}

#if defined(NATIVE_HOST_LIMBS)
__global__ void pad_u64(const uint64_t* __restrict__ src, TestDataTypeUint* __restrict__ dst,
                        size_t L, size_t N, TestDataTypeUint p) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = i < L ? (TestDataTypeUint)(src[i] % p) : (TestDataTypeUint)0;
}
#endif

unsigned grid_for(size_t N) {
    const size_t b = (N + 255) / 256;
    return (unsigned)(b < 148 * 32 ? (b ? b : 1) : 148 * 32);
}
}  // namespace

void zero_pad_gpu(const uint32_t* d_src, TestDataTypeUint* d_dst, size_t L, size_t N,
                  cudaStream_t stream) {
    pad_u32<<<grid_for(N), 256, 0, stream>>>(d_src, d_dst, L, N);
}

#if defined(NATIVE_HOST_LIMBS)
void zero_pad_gpu_u64(const uint64_t* d_src, TestDataTypeUint* d_dst, size_t L, size_t N,
                      TestDataTypeUint modulus, cudaStream_t stream) {
    pad_u64<<<grid_for(N), 256, 0, stream>>>(d_src, d_dst, L, N, modulus);
}
#endif
