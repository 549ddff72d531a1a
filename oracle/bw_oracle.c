/*
 * bw_oracle.c -- CPU restatement of the reference's multiply algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for libbirdwing's
 * CUDA path: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it.  The product path never calls it.
 *
 * Each function names the reference code it restates (paths inside
 * nikitaborisov/birdwing).  The reference's NTT itself comes from the absent
 * GPU-NTT submodule, so the transform follows the reference's own Python
 * model (scripts/full_mul.py:13-63): bit-reversal permutation, iterative
 * radix-2 Cooley-Tukey butterflies with the per-length root
 * w_len = omega^(n/len), and the inverse with omega^-1 and n^-1.  The roots
 * are derived the way the reference derives them: square the table's
 * maximal-order root down to order n (src/gpu_ntt.cu:171-192).
 *
 * Garner follows crt_combine_many (src/crt.cpp:42-87) and the mixed-radix
 * kernel (src/crt_gpu.cu:157-276), with the running value kept in three
 * 64-bit words so that three 64-bit-path primes fit.  Carry propagation follows
 * the serial reference of tests/test_carry_prop.cu:20-35 / scripts/carry.py.
 * The schoolbook product follows tests/test_full_multiply.cpp:27-58.
 *
 * Parity pins: the golden vectors of scripts/full_mul.py:103-124, the CRT
 * known answers of tests/test_crt.cpp and tests/test_crt_gpu.cu, the carry
 * patterns of tests/test_carry_prop.cu and GMP mpz_mul on seeded inputs
 * (tests/golden/).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ---- threads: a plain pthread parallel-for over [0, count) ------------- */

static int g_threads = 1;

/* Number of host threads the oracle may use (1 = serial, the default). */
void oracle_set_threads(int t) { g_threads = t < 1 ? 1 : (t > 256 ? 256 : t); }

typedef void (*range_fn)(size_t lo, size_t hi, void* arg);
typedef struct {
    range_fn fn;
    void* arg;
    size_t lo, hi;
} par_job;

static void* par_run(void* p) {
    par_job* j = (par_job*)p;
    j->fn(j->lo, j->hi, j->arg);
    return NULL;
}

static void par_for(size_t count, size_t min_chunk, range_fn fn, void* arg) {
    int t = g_threads;
    if (t > 1 && count / (size_t)t < min_chunk) t = (int)(count / (min_chunk ? min_chunk : 1));
    if (t <= 1) {
        fn(0, count, arg);
        return;
    }
    pthread_t th[256];
    par_job jobs[256];
    for (int i = 0; i < t; i++) {
        jobs[i].fn = fn;
        jobs[i].arg = arg;
        jobs[i].lo = count * (size_t)i / (size_t)t;
        jobs[i].hi = count * (size_t)(i + 1) / (size_t)t;
    }
    int started = 0;
    for (int i = 1; i < t; i++) {
        if (pthread_create(&th[i], NULL, par_run, &jobs[i]) != 0) break;
        started = i;
    }
    fn(jobs[0].lo, jobs[0].hi, arg);
    for (int i = 1; i <= started; i++) pthread_join(th[i], NULL);
    for (int i = started + 1; i < t; i++) fn(jobs[i].lo, jobs[i].hi, arg);
}

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) { return (uint64_t)((u128)a * b % p); }
static uint64_t addmod(uint64_t a, uint64_t b, uint64_t p) {
    uint64_t s = a + b;  /* a, b < p < 2^63 */
    return s >= p ? s - p : s;
}
static uint64_t submod(uint64_t a, uint64_t b, uint64_t p) { return a >= b ? a - b : a + p - b; }
static uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}
/* Fermat inverse (p prime); the reference uses extended Euclid
 * (modinv_u64, src/crt_utils.cpp:28-50) -- same value. */
static uint64_t invmod(uint64_t a, uint64_t p) { return powmod(a % p, p - 2, p); }

/* ---- limits (src/ntt_limits.cpp:14-61) ------------------------------- */

int oracle_v2(uint64_t x) {
    int k = 0;
    if (x == 0) return 0;
    while ((x & 1) == 0) {
        x >>= 1;
        k++;
    }
    return k;
}

/* largest k with root^(2^k) == 1 reached by squaring, capped at 62
 * (max_root_order, src/ntt_limits.cpp:40-56) */
int oracle_root_order_log(uint64_t root, uint64_t p) {
    uint64_t r = root % p;
    int k = 0;
    if (r == 0) return 0;
    while (k < 62) {
        if (r == 1) return k;
        r = mulmod(r, r, p);
        k++;
    }
    return k;
}

/* root of order 2^log_n from a root of order 2^max_log by repeated squaring
 * (generate_factors_for_N, src/gpu_ntt.cu:184-189) */
uint64_t oracle_root_for(uint64_t p, uint64_t root_max, int max_log, int log_n) {
    uint64_t r = root_max % p;
    for (int j = 0; j < max_log - log_n; j++) r = mulmod(r, r, p);
    return r;
}

/* ---- NTT (scripts/full_mul.py:13-63) ------------------------------------ */

static void bit_reverse_copy(uint64_t* a, size_t n) {
    size_t j = 0;
    for (size_t i = 1; i < n; i++) {
        size_t bit = n >> 1;
        while (j & bit) {
            j ^= bit;
            bit >>= 1;
        }
        j |= bit;
        if (i < j) {
            uint64_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
}

typedef struct {
    uint64_t* a;
    const uint64_t* wp;
    size_t half, len;
    uint64_t p;
} stage_arg;

/* butterflies b in [lo, hi) of one stage: block b / half, offset b % half */
static void stage_range(size_t lo, size_t hi, void* v) {
    const stage_arg* s = (const stage_arg*)v;
    uint64_t* a = s->a;
    const uint64_t p = s->p;
    for (size_t b = lo; b < hi; b++) {
        const size_t j = b % s->half;
        const size_t i = (b / s->half) * s->len;
        const uint64_t u = a[i + j];
        const uint64_t v2_ = mulmod(a[i + j + s->half], s->wp[j], p);
        a[i + j] = addmod(u, v2_, p);
        a[i + j + s->half] = submod(u, v2_, p);
    }
}

static void ntt_core(uint64_t* a, size_t n, uint64_t omega, uint64_t p) {
    bit_reverse_copy(a, n);
    for (size_t len = 2; len <= n; len <<= 1) {
        const uint64_t wlen = powmod(omega, n / len, p);
        const size_t half = len / 2;
        /* powers of wlen for this stage (the Python model advances w
         * serially inside each block; the values are identical) */
        uint64_t* wp = (uint64_t*)malloc(sizeof(uint64_t) * half);
        wp[0] = 1;
        for (size_t j = 1; j < half; j++) wp[j] = mulmod(wp[j - 1], wlen, p);
        stage_arg s = {a, wp, half, len, p};
        par_for(n / 2, 16384, stage_range, &s);
        free(wp);
    }
}

/* forward NTT in place: x_k = sum_i a_i omega^(ik) (natural order out) */
void oracle_ntt(uint64_t* a, size_t n, uint64_t omega, uint64_t p) { ntt_core(a, n, omega, p); }

/* inverse NTT in place, including n^-1 */
void oracle_intt(uint64_t* a, size_t n, uint64_t omega, uint64_t p) {
    ntt_core(a, n, invmod(omega, p), p);
    const uint64_t ninv = invmod(n % p, p);
    for (size_t i = 0; i < n; i++) a[i] = mulmod(a[i], ninv, p);
}

/* cyclic convolution mod (X^n - 1, p) of zero-padded a, b
 * (convolution_mod, scripts/full_mul.py:65-86) */
int oracle_conv_mod(uint64_t p, uint64_t omega_n, const uint64_t* a, size_t la,
                    const uint64_t* b, size_t lb, uint64_t* out, size_t n) {
    if (la > n || lb > n) return -1;
    uint64_t* A = (uint64_t*)calloc(n, sizeof(uint64_t));
    uint64_t* B = (uint64_t*)calloc(n, sizeof(uint64_t));
    if (!A || !B) {
        free(A);
        free(B);
        return -2;
    }
    for (size_t i = 0; i < la; i++) A[i] = a[i] % p;
    for (size_t i = 0; i < lb; i++) B[i] = b[i] % p;
    ntt_core(A, n, omega_n, p);
    ntt_core(B, n, omega_n, p);
    for (size_t i = 0; i < n; i++) A[i] = mulmod(A[i], B[i], p);
    oracle_intt(A, n, omega_n, p);
    memcpy(out, A, n * sizeof(uint64_t));
    free(A);
    free(B);
    return 0;
}

/* ---- Garner (src/crt.cpp:42-87, src/crt_gpu.cu:157-276) ------------------ */

/* x (3 little-endian u64 words, value mod 2^192) from residues r[k] mod
 * primes[k], k < K <= 3: x = k0 + k1 p0 + k2 p0 p1 with mixed-radix digits
 * k_i = (r_i - x mod p_i) * (p0..p_{i-1})^-1 mod p_i. */
int oracle_garner(int K, const uint64_t* primes, const uint64_t* r, uint64_t* x3) {
    uint64_t x[3] = {0, 0, 0};
    uint64_t M[3] = {1, 0, 0}; /* running product of processed primes */
    if (K < 1 || K > 3) return -1;
    for (int i = 0; i < K; i++) {
        const uint64_t p = primes[i];
        /* x mod p and M mod p from the words */
        const uint64_t b64 = powmod(2, 64, p), b128 = mulmod(b64, b64, p);
        uint64_t xm = addmod(addmod(x[0] % p, mulmod(x[1] % p, b64, p), p),
                             mulmod(x[2] % p, b128, p), p);
        uint64_t Mm = addmod(addmod(M[0] % p, mulmod(M[1] % p, b64, p), p),
                             mulmod(M[2] % p, b128, p), p);
        const uint64_t t = submod(r[i] % p, xm, p);
        const uint64_t ki = mulmod(t, invmod(Mm, p), p);
        /* x += M * ki ; M *= p  (mod 2^192) */
        u128 c = 0;
        uint64_t prod[3], Mn[3];
        for (int w = 0; w < 3; w++) {
            u128 s = (u128)M[w] * ki + c;
            prod[w] = (uint64_t)s;
            c = s >> 64;
        }
        c = 0;
        for (int w = 0; w < 3; w++) {
            u128 s = (u128)x[w] + prod[w] + c;
            x[w] = (uint64_t)s;
            c = s >> 64;
        }
        c = 0;
        for (int w = 0; w < 3; w++) {
            u128 s = (u128)M[w] * p + c;
            Mn[w] = (uint64_t)s;
            c = s >> 64;
        }
        memcpy(M, Mn, sizeof M);
    }
    memcpy(x3, x, sizeof x);
    return 0;
}

/* ---- carry (tests/test_carry_prop.cu:20-35, scripts/carry.py:4-21) ------ */

/* out[0..m) = low m words (32-bit) of sum_i c_i 2^(coeff_bits * i), where
 * c_i are 3-word (192-bit) coefficients; coeff_bits is 16 or 32. */
int oracle_carry(const uint64_t* c3, size_t n, int coeff_bits, uint32_t* out, size_t m) {
    /* accumulate in base 2^32 with a 4-word running carry */
    uint64_t acc[4] = {0, 0, 0, 0}; /* value = sum acc[w] 2^(64 w) */
    size_t o = 0;
    if (coeff_bits != 16 && coeff_bits != 32) return -1;
    const int per = 32 / coeff_bits; /* coefficients per output word */
    size_t i = 0;
    while (o < m) {
        for (int q = 0; q < per; q++, i++) {
            if (i >= n) continue;
            const int sh = q * coeff_bits; /* 0 or 16 */
            /* acc += c_i << sh, c_i spread over 4 words after the shift */
            uint64_t s4[4];
            const uint64_t* c = c3 + 3 * i;
            if (sh == 0) {
                s4[0] = c[0];
                s4[1] = c[1];
                s4[2] = c[2];
                s4[3] = 0;
            } else {
                s4[0] = c[0] << sh;
                s4[1] = (c[1] << sh) | (c[0] >> (64 - sh));
                s4[2] = (c[2] << sh) | (c[1] >> (64 - sh));
                s4[3] = c[2] >> (64 - sh);
            }
            u128 cy = 0;
            for (int w = 0; w < 4; w++) {
                const u128 s = (u128)acc[w] + s4[w] + cy;
                acc[w] = (uint64_t)s;
                cy = s >> 64;
            }
        }
        out[o++] = (uint32_t)acc[0];
        /* acc >>= 32 */
        for (int w = 0; w < 4; w++) acc[w] = (acc[w] >> 32) | (w < 3 ? (acc[w + 1] << 32) : 0);
    }
    return 0;
}

/* ---- schoolbook (tests/test_full_multiply.cpp:27-58) --------------------- */

int oracle_schoolbook(const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* out) {
    const size_t n = la + lb;
    u128* tmp = (u128*)calloc(n, sizeof(u128));
    if (!tmp) return -2;
    for (size_t i = 0; i < la; i++)
        for (size_t j = 0; j < lb; j++) tmp[i + j] += (u128)a[i] * b[j];
    u128 carry = 0;
    for (size_t i = 0; i < n; i++) {
        tmp[i] += carry;
        out[i] = (uint32_t)tmp[i];
        carry = tmp[i] >> 32;
    }
    free(tmp);
    return 0;
}

/* ---- full product ---------------------------------------------------------- */

typedef struct {
    int K;
    const uint64_t* primes;
    const uint64_t* res;
    uint64_t* c3;
    size_t n;
} garner_arg;

static void garner_range(size_t lo, size_t hi, void* v) {
    const garner_arg* g = (const garner_arg*)v;
    for (size_t i = lo; i < hi; i++) {
        uint64_t r[3];
        for (int k = 0; k < g->K; k++) r[k] = g->res[(size_t)k * g->n + i];
        oracle_garner(g->K, g->primes, r, g->c3 + 3 * i);
    }
}

/* Product of a (la u32 words) and b (lb words) with an explicit RNS basis:
 * coefficient size coeff_bits (16 or 32), K primes with maximal-order roots.
 * out receives la + lb words. */
int oracle_multiply_basis(int coeff_bits, int K, const uint64_t* primes, const uint64_t* roots_max,
                          const int* max_logs, const uint32_t* a, size_t la, const uint32_t* b,
                          size_t lb, uint32_t* out) {
    const int per = 32 / coeff_bits;
    const size_t na = la * per, nb = lb * per;
    size_t n = 1;
    int log_n = 0;
    while (n < na + nb - 1) {
        n <<= 1;
        log_n++;
    }
    uint64_t* ca = (uint64_t*)malloc(na * sizeof(uint64_t));
    uint64_t* cb = (uint64_t*)malloc(nb * sizeof(uint64_t));
    uint64_t* res = (uint64_t*)malloc((size_t)K * n * sizeof(uint64_t));
    uint64_t* c3 = (uint64_t*)malloc(3 * n * sizeof(uint64_t));
    int rc = 0;
    if (!ca || !cb || !res || !c3) {
        rc = -2;
        goto done;
    }
    for (size_t i = 0; i < na; i++)
        ca[i] = per == 1 ? a[i] : (a[i / 2] >> (16 * (i & 1))) & 0xffff;
    for (size_t i = 0; i < nb; i++)
        cb[i] = per == 1 ? b[i] : (b[i / 2] >> (16 * (i & 1))) & 0xffff;
    for (int k = 0; k < K; k++) {
        if (log_n > max_logs[k]) {
            rc = -3;
            goto done;
        }
        const uint64_t w = oracle_root_for(primes[k], roots_max[k], max_logs[k], log_n);
        rc = oracle_conv_mod(primes[k], w, ca, na, cb, nb, res + (size_t)k * n, n);
        if (rc) goto done;
    }
    {
        garner_arg g = {K, primes, res, c3, n};
        par_for(n, 16384, garner_range, &g);
    }
    rc = oracle_carry(c3, n, coeff_bits, out, la + lb);
done:
    free(ca);
    free(cb);
    free(res);
    free(c3);
    return rc;
}

/* The library's two bases (same primes as libbirdwing), roots derived from a
 * generator of the multiplicative group. */
static const uint64_t P64[3] = {0x3ffffd500000001ull, 0x3ffffcf00000001ull, 0x3ffffa500000001ull};
static const uint64_t G64[3] = {5, 11, 7};
static const uint64_t P32[3] = {469762049ull, 167772161ull, 754974721ull};
static const uint64_t G32[3] = {3, 3, 11};

int oracle_path_basis(int path, uint64_t* primes, uint64_t* roots_max, int* max_logs) {
    const uint64_t* P = path == 64 ? P64 : P32;
    const uint64_t* G = path == 64 ? G64 : G32;
    if (path != 32 && path != 64) return -1;
    for (int k = 0; k < 3; k++) {
        primes[k] = P[k];
        max_logs[k] = oracle_v2(P[k] - 1);
        roots_max[k] = powmod(G[k], (P[k] - 1) >> max_logs[k], P[k]);
    }
    return 0;
}

/* path 32: 16-bit coefficients over the 30-bit primes; path 64: 32-bit
 * coefficients over the 58-bit primes. */
int oracle_multiply(int path, int K, const uint32_t* a, size_t la, const uint32_t* b, size_t lb,
                    uint32_t* out) {
    uint64_t primes[3], roots[3];
    int logs[3];
    if (oracle_path_basis(path, primes, roots, logs)) return -1;
    return oracle_multiply_basis(path == 64 ? 32 : 16, K, primes, roots, logs, a, la, b, lb, out);
}
