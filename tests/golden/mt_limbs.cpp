// Emits std::mt19937_64-generated inputs in the reference's patterns, as raw
// little-endian bytes on stdout.  Used only by gen_golden.py.
//   mt_limbs raw N SEED     -> N successive 64-bit outputs
//   mt_limbs ref32 N SEED   -> tests/test_full_multiply.cpp:61-73 (u32)
//   mt_limbs ref64 N SEED   -> tests/test_full_multiply.cpp:431-441 (u64)
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    const size_t n = strtoull(argv[2], nullptr, 10);
    const uint64_t seed = strtoull(argv[3], nullptr, 10);
    std::mt19937_64 rng(seed);
    if (!strcmp(argv[1], "raw")) {
        std::vector<uint64_t> v(n);
        for (auto& x : v) x = rng();
        fwrite(v.data(), 8, n, stdout);
    } else if (!strcmp(argv[1], "ref32")) {
        std::vector<uint32_t> v(n);
        for (size_t i = 0; i < n; i++) {
            if (i % 8 == 0) v[i] = 0;
            else if (i % 8 == 1) v[i] = 1;
            else v[i] = (uint32_t)rng() % (1ULL << 30);
        }
        fwrite(v.data(), 4, n, stdout);
    } else if (!strcmp(argv[1], "ref64")) {
        std::vector<uint64_t> v(n);
        for (size_t i = 0; i < n; i++) {
            if (i % 8 == 0) v[i] = 0;
            else if (i % 8 == 1) v[i] = 1;
            else if (i % 8 == 2) v[i] = UINT64_MAX;
            else v[i] = rng();
        }
        fwrite(v.data(), 8, n, stdout);
    } else {
        return 2;
    }
    return 0;
}
