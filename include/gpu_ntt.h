// gpu_ntt.h -- multiply lifecycle (precompute / upload / allocate / execute /
// cleanup), compatible with nikitaborisov/birdwing include/gpu_ntt.h:18-118.
// The reference builds these on the GPU-NTT library; here they are shims over
// libbirdwing's C ABI (bw_plan / bw_ctx, birdwing.h), implemented in
// birdwing_b200/csrc/compat/gpu_ntt.cu.  Structs keep the fields callers
// read (N, logN, the timing structs field for field); the GPU-NTT internals
// (params, Root/Modulus tables) have no counterpart.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "birdwing.h"
#include "carry_prop.h"
#include "config.h"
#include "crt_gpu.h"

using namespace std;

typedef TestDataTypeUint TestDataType;

struct NTTContext {
    size_t N = 0;  // padded transform length in limbs (next_pow2(L_A + L_B - 1))
    int logN = 0;
    size_t L_A = 0, L_B = 0;
    cudaStream_t stream_a = nullptr;  // the stream all work is issued on
    cudaStream_t stream_b = nullptr;  // same stream (kept for source compatibility)
    bw_plan* plan = nullptr;
    bw_ctx* ctx = nullptr;
};

struct NTTPrecomputed {
    size_t N = 0;
    int logN = 0;
    CRTGarnerParams garner{};
    bool gpu_uploaded = false;
};

struct PrecomputeTiming {
    float factors_ms = 0.0f;
    float params_ms = 0.0f;
    float twiddle_host_ms = 0.0f;
    float garner_host_ms = 0.0f;
    float total_ms = 0.0f;
};

struct SetupUploadTiming {
    float twiddle_upload_ms = 0.0f;
    float mod_constants_ms = 0.0f;
    float garner_upload_ms = 0.0f;
    float total_ms = 0.0f;
};

// Stage times (ms, CUDA events).  libbirdwing fuses stages: fwd_pad_ntt_* is
// limb split + pad + forward column pass of both operands, pointwise_mul_ms
// the fused row pass (forward rows, product, inverse rows), intt_ms the
// inverse column pass, crt_ms the fused Garner + carry, carry_ms 0.
struct NTTTiming {
    float ingress_fwd_ms = 0.0f;
    float h2d_ms = 0.0f;
    float fwd_pad_ntt_ms = 0.0f;
    float fwd_pad_ntt_a_ms = 0.0f;
    float fwd_pad_ntt_b_ms = 0.0f;
    float pointwise_mul_ms = 0.0f;
    float intt_ms = 0.0f;
    float crt_ms = 0.0f;
    float carry_ms = 0.0f;
    float d2h_ms = 0.0f;
    float total_ms = 0.0f;
};

NTTPrecomputed precompute_ntt(size_t N, PrecomputeTiming* timing_out = nullptr);
void upload_ntt_precomputed(NTTPrecomputed& pre, SetupUploadTiming* timing_out = nullptr);
NTTContext allocate_ntt_context(const NTTPrecomputed& pre, size_t L_A, size_t L_B);

// C_out must hold at least L_A + L_B limbs (the reference requires N + 1);
// limbs from L_A + L_B on are set to 0.  With crt_hi_out/crt_lo_out (u32-limb
// widths) the call returns the n convolution coefficients before carry.
void execute_ntt_multiply(NTTContext& ctx, const InputLimbType* a_pinned,
                          const InputLimbType* b_pinned, vector<OutputLimbType>& C_out,
                          NTTTiming* timing_out = nullptr, vector<uint64_t>* crt_hi_out = nullptr,
                          vector<uint64_t>* crt_lo_out = nullptr,
                          vector<uint64_t>* crt_mid_out = nullptr,
                          vector<uint32_t>* crt_hi32_out = nullptr);

void cleanup_ntt_context(NTTContext& ctx);
void cleanup_ntt_precomputed(NTTPrecomputed& pre);
