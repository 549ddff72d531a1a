// bw_host.h -- internal host helpers shared by the library's translation units.
#pragma once
#include <cstddef>
#include <cstdint>

// Record a message for bw_last_error() and return code.
int bw_fail(int code, const char* fmt, ...);
void bw_clear_error();

// Admission check of one product size on one path (BW_OK or BW_ESIZE).
int bw_check_size(int path, int num_primes, size_t la, size_t lb, int* log_n_out);

// Largest transform length (log2) a path supports with K primes.
int bw_path_max_log_n(int path, int num_primes);

// The path's primes (three entries).
const uint64_t* bw_path_primes(int path);

// The path BW_PATH_AUTO picks for a product of la x lb words with K primes
// (w64_ok: the 64-bit path would use 64-bit coefficients, single products
// with num_primes 0).
int bw_choose_path(int K, size_t la, size_t lb, bool w64_ok = false);
