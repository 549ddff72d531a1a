// carry_prop.cu -- the reference's three-kernel segmented carry with its
// launch protocol (src/carry_prop.cu:8-211, host loop src/gpu_ntt.cu:889-924):
//   intra <<<num_segs, 1>>>  each segment resolved serially with carry-in 0
//   inter <<<1, 1>>>         seg_carry becomes the carry INTO each segment
//   fixup <<<num_segs, 1>>>  repeated by the host while *escape_flag is set
// The fixup consumes its segment's incoming carry with an atomic exchange, so
// a carry that escapes a segment is applied exactly once even across
// repeated launches.  128-bit coefficients keep signed 64-bit segment
// carries (the reference's storage type); 160-bit ones keep three words.
#include <cuda_runtime.h>

#include "carry_prop.h"

namespace {
constexpr int kShift = OUTPUT_LIMB_BITS;
__device__ __forceinline__ size_t seg_end(size_t s, size_t N) {
    const size_t e = (s + 1) * CARRY_SEG;
    return e < N ? e : N;
}
}  // namespace

__global__ void carry_intra_segment_kernel(const uint64_t* __restrict__ C_hi,
                                           const uint64_t* __restrict__ C_lo,
                                           OutputLimbType* __restrict__ out,
                                           int64_t* __restrict__ seg_carry, size_t N) {
    if (threadIdx.x != 0) return;
    const size_t s = blockIdx.x;
    unsigned __int128 c = 0;
    for (size_t i = s * CARRY_SEG; i < seg_end(s, N); ++i) {
        const unsigned __int128 v = (((unsigned __int128)C_hi[i] << 64) | C_lo[i]) + c;
        out[i] = (OutputLimbType)v;
        c = v >> kShift;
    }
    seg_carry[s] = (int64_t)c;
}

__global__ void carry_inter_segment_kernel(int64_t* __restrict__ seg_carry, size_t num_segs) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t prev = 0;
    for (size_t s = 0; s < num_segs; ++s) {
        const int64_t own = seg_carry[s];
        seg_carry[s] = prev;
        prev = own;
    }
}

__global__ void carry_fixup_kernel(OutputLimbType* __restrict__ out,
                                   int64_t* __restrict__ seg_carry, size_t N, size_t num_segs,
                                   int* __restrict__ escape_flag) {
    if (threadIdx.x != 0) return;
    const size_t s = blockIdx.x;
    unsigned long long* slot = reinterpret_cast<unsigned long long*>(&seg_carry[s]);
    unsigned __int128 c = (uint64_t)atomicExch(slot, 0ull);
    for (size_t i = s * CARRY_SEG; i < seg_end(s, N) && c != 0; ++i) {
        const unsigned __int128 v = (unsigned __int128)out[i] + c;
        out[i] = (OutputLimbType)v;
        c = v >> kShift;
    }
    if (c != 0 && s + 1 < num_segs) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&seg_carry[s + 1]),
                  (unsigned long long)(uint64_t)c);
        *escape_flag = 1;
    }
}

#if defined(NATIVE_HOST_LIMBS)

namespace {
// (lo, mid, hi) 160-bit helpers
struct W160 {
    uint64_t lo, mid;
    uint32_t hi;
};
__device__ __forceinline__ W160 add160(W160 a, W160 b) {
    const unsigned __int128 s0 = (unsigned __int128)a.lo + b.lo;
    const unsigned __int128 s1 = (unsigned __int128)a.mid + b.mid + (uint64_t)(s0 >> 64);
    return W160{(uint64_t)s0, (uint64_t)s1, a.hi + b.hi + (uint32_t)(s1 >> 64)};
}
__device__ __forceinline__ bool nz(const W160& a) { return a.lo | a.mid | a.hi; }
}  // namespace

__global__ void carry_intra_segment_kernel_u160(const uint64_t* __restrict__ C_lo,
                                                const uint64_t* __restrict__ C_mid,
                                                const uint32_t* __restrict__ C_hi,
                                                OutputLimbType* __restrict__ out,
                                                uint64_t* __restrict__ seg_carry_lo,
                                                uint64_t* __restrict__ seg_carry_mid,
                                                uint32_t* __restrict__ seg_carry_hi, size_t N) {
    if (threadIdx.x != 0) return;
    const size_t s = blockIdx.x;
    W160 c{0, 0, 0};
    for (size_t i = s * CARRY_SEG; i < seg_end(s, N); ++i) {
        const W160 v = add160(W160{C_lo[i], C_mid[i], C_hi[i]}, c);
        out[i] = (OutputLimbType)v.lo;
        c = W160{v.mid, (uint64_t)v.hi, 0};  // v >> 64
    }
    seg_carry_lo[s] = c.lo;
    seg_carry_mid[s] = c.mid;
    seg_carry_hi[s] = c.hi;
}

__global__ void carry_inter_segment_kernel_u160(uint64_t* __restrict__ seg_carry_lo,
                                                uint64_t* __restrict__ seg_carry_mid,
                                                uint32_t* __restrict__ seg_carry_hi,
                                                size_t num_segs) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    W160 prev{0, 0, 0};
    for (size_t s = 0; s < num_segs; ++s) {
        const W160 own{seg_carry_lo[s], seg_carry_mid[s], seg_carry_hi[s]};
        seg_carry_lo[s] = prev.lo;
        seg_carry_mid[s] = prev.mid;
        seg_carry_hi[s] = prev.hi;
        prev = own;
    }
}

__global__ void carry_fixup_kernel_u160(OutputLimbType* __restrict__ out,
                                        uint64_t* __restrict__ seg_carry_lo,
                                        uint64_t* __restrict__ seg_carry_mid,
                                        uint32_t* __restrict__ seg_carry_hi, size_t N,
                                        size_t num_segs, int* __restrict__ escape_flag) {
    if (threadIdx.x != 0) return;
    const size_t s = blockIdx.x;
    W160 c{(uint64_t)atomicExch(reinterpret_cast<unsigned long long*>(&seg_carry_lo[s]), 0ull),
           (uint64_t)atomicExch(reinterpret_cast<unsigned long long*>(&seg_carry_mid[s]), 0ull),
           atomicExch(reinterpret_cast<unsigned int*>(&seg_carry_hi[s]), 0u)};
    for (size_t i = s * CARRY_SEG; i < seg_end(s, N) && nz(c); ++i) {
        const W160 v = add160(W160{out[i], 0, 0}, c);
        out[i] = (OutputLimbType)v.lo;
        c = W160{v.mid, (uint64_t)v.hi, 0};
    }
    if (nz(c) && s + 1 < num_segs) {
        // multi-word atomic add into the next segment's carry
        const unsigned long long old_lo = atomicAdd(
            reinterpret_cast<unsigned long long*>(&seg_carry_lo[s + 1]), (unsigned long long)c.lo);
        const uint64_t cy0 = (old_lo + c.lo < old_lo) ? 1u : 0u;
        const unsigned __int128 m = (unsigned __int128)c.mid + cy0;
        const uint64_t add_mid = (uint64_t)m;
        const unsigned long long old_mid = atomicAdd(
            reinterpret_cast<unsigned long long*>(&seg_carry_mid[s + 1]), add_mid);
        const uint32_t cy1 = ((old_mid + add_mid < old_mid) ? 1u : 0u) + (uint32_t)(m >> 64);
        if (c.hi + cy1) atomicAdd(reinterpret_cast<unsigned int*>(&seg_carry_hi[s + 1]), c.hi + cy1);
        *escape_flag = 1;
    }
}

#endif  // NATIVE_HOST_LIMBS
