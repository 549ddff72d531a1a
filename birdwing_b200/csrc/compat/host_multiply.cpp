// host_multiply.cpp -- the reference's one-shot product over the C ABI.
// Reference: host_multiply_merge / _native, src/host_multiply.cpp:27-134
// (admission failures print and exit(1) there; the same here).
#include <chrono>
#include <cstdio>
#include <cstdlib>

#include "birdwing.h"
#include "multiply.h"

namespace {
void run(const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* c, size_t lc,
         chrono::duration<double, milli>& duration) {
    const auto t0 = chrono::high_resolution_clock::now();
    float ms = 0.f;
    if (bw_multiply_host_once(a, la, b, lb, c, lc, BW_PATH_AUTO, &ms) != BW_OK) {
        fprintf(stderr, "[NTT] Unsupported multiply: %s\n", bw_last_error());
        exit(1);
    }
    duration = chrono::high_resolution_clock::now() - t0;
}
}  // namespace

#if !defined(NATIVE_HOST_LIMBS)
void host_multiply_merge(const vector<uint32_t>& A, const vector<uint32_t>& B,
                         vector<OutputLimbType>& C, chrono::duration<double, milli>& duration) {
    C.assign(A.size() + B.size(), 0);
    run(A.data(), A.size(), B.data(), B.size(), reinterpret_cast<uint32_t*>(C.data()), C.size(),
        duration);
}
#endif

#if defined(NATIVE_HOST_LIMBS)
void host_multiply_merge_native(const vector<uint64_t>& A, const vector<uint64_t>& B,
                                vector<uint64_t>& C, chrono::duration<double, milli>& duration) {
    C.assign(A.size() + B.size(), 0);
    run(reinterpret_cast<const uint32_t*>(A.data()), 2 * A.size(),
        reinterpret_cast<const uint32_t*>(B.data()), 2 * B.size(),
        reinterpret_cast<uint32_t*>(C.data()), 2 * C.size(), duration);
}
#endif
