// gpu_ntt.cpp -- the reference's multiply lifecycle over libbirdwing's C ABI.
// Compiled with the caller's width macros (see include/config.h).
//
// Reference: src/gpu_ntt.cu:240-1018 (precompute_ntt .. cleanup_*).
#include "gpu_ntt.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ntt_limits.h"

// RNS tables of this width: libbirdwing's primes with maximal-order roots.
#if LIMB_BITS == 64 && defined(NATIVE_HOST_LIMBS)
vector<TestDataTypeUint> moduli = {0x3ffffd500000001ULL, 0x3ffffcf00000001ULL,
                                   0x3ffffa500000001ULL};
vector<TestDataTypeUint> roots_of_unity_max = {0, 0, 0};
#elif LIMB_BITS == 64
vector<TestDataTypeUint> moduli = {0x3ffffd500000001ULL, 0x3ffffcf00000001ULL};
vector<TestDataTypeUint> roots_of_unity_max = {0, 0};
#else
vector<TestDataTypeUint> moduli = {469762049u, 167772161u, 754974721u};
vector<TestDataTypeUint> roots_of_unity_max = {0, 0, 0};
#endif

namespace {

// the path the lifecycle drives: 58-bit primes (u32 coefficients); the CRT
// coefficients it can dump are then those of the limb-level convolution
constexpr int kPath = BW_PATH_P64;
constexpr int kWordsPerLimb = INPUT_LIMB_BITS / 32;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) {
    return (uint64_t)((unsigned __int128)a * b % p);
}
uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

// generator of the multiplicative group of each library prime
uint64_t generator(uint64_t p) {
    switch (p) {
        case 0x3ffffd500000001ULL: return 5;
        case 0x3ffffcf00000001ULL: return 11;
        case 0x3ffffa500000001ULL: return 7;
        case 754974721u: return 11;
        case 469762049u: return 3;
        case 167772161u: return 3;
        default: return 0;
    }
}

// fill roots_of_unity_max from the generators (once)
struct RootsInit {
    RootsInit() {
        for (size_t i = 0; i < moduli.size(); ++i) {
            const uint64_t p = moduli[i];
            int v = 0;
            uint64_t t = p - 1;
            while ((t & 1) == 0) {
                t >>= 1;
                ++v;
            }
            roots_of_unity_max[i] = (TestDataTypeUint)powmod(generator(p), (p - 1) >> v, p);
        }
    }
} g_roots_init;

[[noreturn]] void die(const char* what) {
    fprintf(stderr, "[NTT] %s: %s\n", what, bw_last_error());
    exit(1);
}

}  // namespace

NTTPrecomputed precompute_ntt(size_t N, PrecomputeTiming* timing_out) {
    const auto t0 = chrono::high_resolution_clock::now();
    NTTPrecomputed pre;
    if (N == 0 || (N & (N - 1))) {
        fprintf(stderr, "[NTT] Unsupported size: NTT size N=%zu is not a power of two\n", N);
        exit(1);
    }
    pre.N = N;
    pre.logN = 0;
    while (((size_t)1 << pre.logN) < N) ++pre.logN;
    // the library builds its per-size tables when the context is allocated
    // (the transform length depends on L_A and L_B); only Garner constants
    // are host-side here
    pre.garner = compute_garner_params(moduli);
    if (timing_out) {
        memset(timing_out, 0, sizeof *timing_out);
        timing_out->total_ms =
            chrono::duration<float, milli>(chrono::high_resolution_clock::now() - t0).count();
        timing_out->garner_host_ms = timing_out->total_ms;
    }
    return pre;
}

void upload_ntt_precomputed(NTTPrecomputed& pre, SetupUploadTiming* timing_out) {
    if (timing_out) memset(timing_out, 0, sizeof *timing_out);
    pre.gpu_uploaded = true;
}

NTTContext allocate_ntt_context(const NTTPrecomputed& pre, size_t L_A, size_t L_B) {
    if (!pre.gpu_uploaded) {
        fprintf(stderr, "[NTT] allocate_ntt_context: call upload_ntt_precomputed first\n");
        exit(1);
    }
    NTTContext ctx;
    ctx.N = pre.N;
    ctx.logN = pre.logN;
    ctx.L_A = L_A;
    ctx.L_B = L_B;
    if (bw_plan_create(&ctx.plan, kPath, L_A * kWordsPerLimb, L_B * kWordsPerLimb, NUM_MODULI,
                       0) != BW_OK)
        die("allocate_ntt_context");
    if (bw_ctx_create(&ctx.ctx, ctx.plan, nullptr) != BW_OK) die("allocate_ntt_context");
    ctx.stream_a = ctx.stream_b = (cudaStream_t)bw_ctx_stream(ctx.ctx);
    return ctx;
}

void execute_ntt_multiply(NTTContext& ctx, const InputLimbType* a_pinned,
                          const InputLimbType* b_pinned, vector<OutputLimbType>& C_out,
                          NTTTiming* timing_out, vector<uint64_t>* crt_hi_out,
                          vector<uint64_t>* crt_lo_out, vector<uint64_t>* crt_mid_out,
                          vector<uint32_t>* crt_hi32_out) {
    const size_t la = ctx.L_A * kWordsPerLimb, lb = ctx.L_B * kWordsPerLimb;
    const uint32_t* a = reinterpret_cast<const uint32_t*>(a_pinned);
    const uint32_t* b = reinterpret_cast<const uint32_t*>(b_pinned);
#if defined(NATIVE_HOST_LIMBS)
    if (crt_lo_out && crt_mid_out && crt_hi32_out) {
        // the native width's CRT values are coefficients of the u64-limb
        // convolution (up to 160 bits); the library convolves u32 words
        fprintf(stderr, "[NTT] CRT dump of the native-limb width is not supported\n");
        crt_lo_out->clear();
        crt_mid_out->clear();
        crt_hi32_out->clear();
        return;
    }
#else
    (void)crt_mid_out;
    (void)crt_hi32_out;
    if (crt_hi_out && crt_lo_out) {
        bw_plan_info info;
        bw_plan_get_info(ctx.plan, &info);
        const size_t n = (size_t)1 << info.log_n;
        vector<uint32_t> words(3 * n);
        if (bw_multiply_coeffs(ctx.ctx, a, la, b, lb, words.data(), words.size()) != BW_OK)
            die("execute_ntt_multiply");
        crt_hi_out->assign(ctx.N, 0);
        crt_lo_out->assign(ctx.N, 0);
        for (size_t i = 0; i < ctx.N && i < n; ++i) {
            (*crt_lo_out)[i] = (uint64_t)words[3 * i] | ((uint64_t)words[3 * i + 1] << 32);
            (*crt_hi_out)[i] = words[3 * i + 2];
        }
        if (timing_out) memset(timing_out, 0, sizeof *timing_out);
        return;
    }
#endif
    const size_t limbs = ctx.L_A + ctx.L_B;
    if (C_out.size() < limbs) C_out.resize(limbs);
    bw_timing t{};
    if (bw_multiply(ctx.ctx, a, la, b, lb, reinterpret_cast<uint32_t*>(C_out.data()),
                    limbs * kWordsPerLimb, BW_PTR_HOST, timing_out ? &t : nullptr) != BW_OK)
        die("execute_ntt_multiply");
    for (size_t i = limbs; i < C_out.size(); ++i) C_out[i] = 0;
    if (timing_out) {
        timing_out->h2d_ms = t.h2d_ms;
        timing_out->fwd_pad_ntt_ms = timing_out->fwd_pad_ntt_a_ms = timing_out->fwd_pad_ntt_b_ms =
            t.fwd_ms;
        timing_out->ingress_fwd_ms = t.h2d_ms + t.fwd_ms;
        timing_out->pointwise_mul_ms = t.mul_ms;
        timing_out->intt_ms = t.intt_ms;
        timing_out->crt_ms = t.crt_carry_ms;
        timing_out->carry_ms = 0.0f;
        timing_out->d2h_ms = t.d2h_ms;
        timing_out->total_ms = t.total_ms;
    }
}

void cleanup_ntt_context(NTTContext& ctx) {
    bw_ctx_destroy(ctx.ctx);
    bw_plan_destroy(ctx.plan);
    ctx.ctx = nullptr;
    ctx.plan = nullptr;
}

void cleanup_ntt_precomputed(NTTPrecomputed& pre) { pre.gpu_uploaded = false; }
