// ref_stage_shim.cu -- C entry points around the reference's own stage
// kernels (src/crt_gpu.cu and src/carry_prop.cu compiled with LIMB_BITS=64,
// the reference's "hybrid" pipeline: u32 limbs, two 64-bit primes), so that
// parity tests can run them on the GPU beside libbirdwing.  TEST
// INFRASTRUCTURE ONLY; built by build_ref.sh into _ref/libref_stage_hybrid.so.
#include <cuda_runtime.h>

#include "carry_prop.h"
#include "crt_gpu.h"

// declared by the reference's config.h; its stage kernels do not read them
vector<TestDataTypeUint> moduli;
vector<TestDataTypeUint> roots_of_unity_max;

// Garner of two residue arrays (device, n entries each) with the reference's
// crt_combine_gpu (src/crt_gpu.cu:157-203, 293-302).
extern "C" int ref_crt_combine_hybrid(uint64_t p0, uint64_t p1, const uint64_t* d_res0,
                                      const uint64_t* d_res1, int n, uint64_t* d_hi,
                                      uint64_t* d_lo) {
    const vector<TestDataTypeUint> primes = {p0, p1};
    upload_garner_params(compute_garner_params(primes));
    upload_residue_ptrs({const_cast<uint64_t*>(d_res0), const_cast<uint64_t*>(d_res1)});
    crt_combine_gpu(d_hi, d_lo, n);
    return (int)cudaGetLastError();
}

// The reference's three-kernel carry with its host loop (src/gpu_ntt.cu:
// 889-924): 128-bit coefficients (hi, lo) -> n u32 words.  The fixup loop
// is bounded at 64 launches.
extern "C" int ref_carry_hybrid(const uint64_t* d_hi, const uint64_t* d_lo, size_t n,
                                uint32_t* d_out) {
    const size_t segs = (n + CARRY_SEG - 1) / CARRY_SEG;
    int64_t* seg = nullptr;
    int* esc = nullptr;
    if (cudaMalloc(&seg, segs * sizeof(int64_t)) != cudaSuccess) return -1;
    if (cudaMalloc(&esc, sizeof(int)) != cudaSuccess) return -1;
    carry_intra_segment_kernel<<<(unsigned)segs, 1>>>(d_hi, d_lo, d_out, seg, n);
    carry_inter_segment_kernel<<<1, 1>>>(seg, segs);
    int rc = 0;
    for (int it = 0; it < 64; ++it) {
        cudaMemset(esc, 0, sizeof(int));
        carry_fixup_kernel<<<(unsigned)segs, 1>>>(d_out, seg, n, segs, esc);
        int e = 0;
        cudaMemcpy(&e, esc, sizeof(int), cudaMemcpyDeviceToHost);
        if (!e) break;
        if (it == 63) rc = -2;
    }
    cudaFree(seg);
    cudaFree(esc);
    const cudaError_t e = cudaDeviceSynchronize();
    return e != cudaSuccess ? (int)e : rc;
}
