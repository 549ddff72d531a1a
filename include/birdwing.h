/*
 * birdwing.h -- C ABI of the B200-native big-integer multiply library
 * (libbirdwing.so).
 *
 * Multiplies large unsigned integers given as little-endian arrays of 32-bit
 * words ("limbs") with a residue-number-system NTT pipeline on one NVIDIA
 * B200 (sm_100a):
 *
 *   limb split + zero pad -> forward NTT per prime -> pointwise product ->
 *   inverse NTT -> Garner CRT reconstruction -> carry propagation.
 *
 * Two prime paths are compiled into the same library and chosen at run time:
 *
 *   BW_PATH_P32 : 16-bit coefficients, 30-bit primes, 32-bit modular
 *                 arithmetic (the reference's LIMB_BITS=32 pipeline, whose
 *                 transform length is twice the limb count).
 *   BW_PATH_P64 : 32-bit coefficients, 58-bit primes of the form c*2^32+1,
 *                 64-bit modular arithmetic (the reference's LIMB_BITS=64
 *                 "hybrid" and NATIVE_HOST_LIMBS pipelines; a u64 limb array
 *                 is passed as twice as many u32 words).
 *
 * Everything crossing this boundary is a plain pointer, size or POD struct.
 * Every call returns an int status (BW_OK == 0, negative on error); the
 * library never calls exit().  bw_last_error() returns a thread-local
 * message for the most recent failure on the calling thread.
 *
 * Reference interfaces this ABI replaces (paths inside nikitaborisov/birdwing):
 *   host_multiply_merge / host_multiply_merge_native  include/multiply.h:9-23,
 *       src/host_multiply.cpp:27-134              -> bw_multiply_host_once
 *   precompute_ntt + upload_ntt_precomputed           include/gpu_ntt.h:101-102,
 *       src/gpu_ntt.cu:240-379                      -> bw_plan_create
 *   allocate_ntt_context                              include/gpu_ntt.h:103,
 *       src/gpu_ntt.cu:382-440                      -> bw_ctx_create
 *   execute_ntt_multiply                              include/gpu_ntt.h:105-115,
 *       src/gpu_ntt.cu:442-973                      -> bw_multiply / bw_square
 *   execute_ntt_multiply(..., crt_*_out)              src/gpu_ntt.cu:843-884
 *                                                   -> bw_multiply_coeffs
 *   cleanup_ntt_context / cleanup_ntt_precomputed     include/gpu_ntt.h:117-118
 *                                                   -> bw_ctx_destroy / bw_plan_destroy
 *   ntt_limits family                                 include/ntt_limits.h:9-31,
 *       src/ntt_limits.cpp:14-280                   -> bw_limits
 *   NTTTiming                                         include/gpu_ntt.h:87-99
 *                                                   -> bw_timing
 */
#ifndef BIRDWING_H
#define BIRDWING_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BW_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
#define BW_OK            0
#define BW_EINVAL      (-1)  /* bad argument (null pointer, zero length, ...) */
#define BW_ENOMEM      (-2)  /* device or pinned-host allocation failed       */
#define BW_ECUDA       (-3)  /* a CUDA runtime call failed                    */
#define BW_ETIMEOUT    (-4)  /* a bounded device-side wait gave up            */
#define BW_EREJECT     (-5)  /* admission rejected (memory budget)            */
#define BW_ESIZE       (-6)  /* product size outside the supported limits     */
#define BW_ECHECK      (-7)  /* redundant-prime consistency check failed      */
#define BW_EBUSY       (-8)  /* resource still in use                         */

/* ---- prime paths --------------------------------------------------------- */
#define BW_PATH_AUTO   0
#define BW_PATH_P32    32
#define BW_PATH_P64    64

/* ---- flags for bw_plan_create --------------------------------------------- */
/* Split the transform into rows x 2^x columns for the 4-step schedule
 * (0 = automatic).  x <= 13 (64-bit path) or 14 (32-bit path). */
#define BW_PLAN_LOG_COLS(x) (((unsigned)(x) & 0x1fu) << 8)
/* Tuning switches: radix-8 instead of radix-16 rounds in the row pass;
 * stage the column stage twiddles in shared memory (when <= 32 KiB) instead
 * of reading them through L1; use the three-pass schedule (n = R * R2 * C)
 * even where two passes fit (it is used anyway beyond n = 2^26). */
#define BW_PLAN_RADIX8      (1u << 16)
#define BW_PLAN_TW_SMEM     (1u << 17)
#define BW_PLAN_THREE_PASS  (1u << 18)
/* Column-pass tiles of up to 128 KiB of residues instead of 64 KiB (twice
 * the columns per CTA: longer contiguous row segments, fewer CTAs per SM). */
#define BW_PLAN_WIDE_COLS   (1u << 19)
/* 64-bit coefficients (two words each).  On the 64-bit path: three primes,
 * all three carrying the coefficients (no redundant prime), half the
 * transform length of 32-bit coefficients for 1.5x the primes; num_primes 0
 * there chooses it where it halves a transform of at least 2^19 points.  On
 * the 32-bit path: six primes below 2^30 (transforms of up to 2^23 points,
 * operands up to 2^23 words), a quarter of the 16-bit coefficients' transform
 * length for 3x the primes.  With this flag num_primes must be 0, or 3 (64-bit
 * path) or 6 (32-bit path).  The reference splits operands into 32-bit
 * coefficients only (src/zero_pad.cu:3-57); the product is the same. */
#define BW_PLAN_COEF64      (1u << 20)
/* Radix-16 rounds in the row pass where radix 8 is the default (single
 * products on the 64-bit path with rows of at most 2^12 points). */
#define BW_PLAN_RADIX16     (1u << 21)
/* Radix-8 rounds in the column passes (single products on the 64-bit path). */
#define BW_PLAN_COL_RADIX8  (1u << 22)
/* Single products, two-pass schedule: the inverse column pass brings its tile
 * into shared memory with tensor-memory-accelerator box copies
 * (cp.async.bulk.tensor, one mbarrier) instead of per-element cp.async, and
 * runs its rounds on the dense tile.  On by default from transforms of 2^20
 * points (measured faster there, slower below); BW_PLAN_TMA_COLS forces it
 * on, BW_PLAN_NO_TMA_COLS off. */
#define BW_PLAN_TMA_COLS    (1u << 23)
#define BW_PLAN_NO_TMA_COLS (1u << 24)
/* Single products on the 32-bit path with 2^12-point rows: the row pass hands
 * one round's outputs to the next through warp shuffles (a 16 x 16 transpose
 * inside each half-warp) instead of shared memory.  A measured alternative,
 * off by default. */
#define BW_PLAN_SHFL_ROWS   (1u << 25)
/* 32-bit path with 64-bit coefficients: the forward column pass runs one
 * prime per CTA, reducing the coefficients straight into its residue tile,
 * instead of looping over the six primes in one CTA with a u64 copy of the
 * tile's coefficients beside its residues (the default, measured faster). */
#define BW_PLAN_K1_ONE_PRIME (1u << 26)

/* ---- flags for bw_multiply ------------------------------------------------ */
#define BW_PTR_HOST    0u    /* a, b, c are host pointers (pinned or pageable):
                                the call copies in, computes, copies out and
                                synchronises                                 */
#define BW_PTR_DEVICE  1u    /* a, b, c are device pointers: the call only
                                enqueues work on the context's stream        */
#define BW_PTR_HOST_ASYNC 2u /* a, b, c are host pointers (pinned, for the
                                copies to be asynchronous): the call enqueues
                                copy-in, product and copy-out on the context's
                                stream and returns; the buffers must stay
                                valid until bw_ctx_sync, which also reports
                                device-side errors.  Two or three contexts of
                                one plan used in turn overlap one product's
                                copies with another's kernels: host-pointer
                                products of a plan with several live contexts
                                run each stage (copy-in, kernels, copy-out)
                                after the same stage of the plan's previous
                                product.  timing must be NULL.               */

/* Opaque handles.  A plan owns the per-size device tables (twiddles, Garner
 * constants); a context owns device scratch and a stream and borrows its
 * plan's tables (the reference's NTTContext borrows NTTPrecomputed's device
 * pointers the same way, src/gpu_ntt.cu:398-402).  Distinct handles may be
 * used from distinct threads; one context is used by one thread at a time. */
typedef struct bw_plan bw_plan;
typedef struct bw_ctx bw_ctx;

/* Per-stage device times in milliseconds (CUDA events on the context stream).
 * Field meanings follow the reference's NTTTiming (include/gpu_ntt.h:87-99):
 * fwd_ms covers limb split + zero pad + forward column pass for both operands;
 * mul_ms the fused row pass (forward rows, pointwise product, inverse rows);
 * intt_ms the inverse column pass; crt_carry_ms the fused Garner + carry. */
typedef struct bw_timing {
    float h2d_ms;
    float fwd_ms;
    float mul_ms;
    float intt_ms;
    float crt_carry_ms;
    float d2h_ms;
    float total_ms;
} bw_timing;

typedef struct bw_plan_info {
    int      path;          /* BW_PATH_P32 or BW_PATH_P64                    */
    int      num_primes;    /* K                                             */
    int      log_n;         /* transform length n = 2^log_n                  */
    int      log_rows;      /* 4-step split n = rows * cols                   */
    int      log_cols;
    int      coeff_bits;    /* 16, 32 or 64 (BW_PLAN_COEF64)                 */
    size_t   la, lb;        /* operand lengths in u32 words                  */
    size_t   lc;            /* product length in u32 words (= la + lb)       */
    size_t   plan_device_bytes;   /* twiddle + constant tables               */
    size_t   ctx_device_bytes;    /* scratch one context allocates           */
    uint64_t primes[6];     /* the first num_primes entries are set          */
} bw_plan_info;

typedef struct bw_limits_info {
    int      path;
    int      num_primes;
    int      max_log_n;        /* largest transform length supported         */
    size_t   max_square_words; /* largest la == lb (u32 words)               */
} bw_limits_info;

/* Returns BW_ABI_VERSION. */
int bw_abi_version(void);

/* Message describing the last failure on this thread ("" if none). */
const char* bw_last_error(void);

/* Limits of one prime path.  num_primes = 0 selects the default K. */
int bw_limits(int path, int num_primes, bw_limits_info* out);

/* Would a product of la x lb u32 words be accepted?  Returns BW_OK or
 * BW_ESIZE with a reason in bw_last_error().  (Reference:
 * multiply_size_supported, src/ntt_limits.cpp:232-245.) */
int bw_size_supported(int path, int num_primes, size_t la, size_t lb);

/* Build the plan (twiddle tables on the device, Garner constants) for
 * products of la x lb u32 words.  num_primes = 0 lets the library choose:
 * with path = BW_PATH_AUTO, the 32-bit path with 16-bit coefficients (K = 2)
 * while its transform has at most 2^21 points (operands up to about 2^24
 * bits), then the 32-bit path with 64-bit coefficients (K = 6) while its
 * transform has at most 2^23 points (operands up to 2^28 bits), the 64-bit
 * path beyond; on the 64-bit path, 64-bit coefficients with K = 3
 * (BW_PLAN_COEF64) where they halve the transform and it has at least 2^19
 * points, else 32-bit coefficients with K = 2.  num_primes 2 or 3 keeps the
 * reference's 16- or 32-bit coefficients (and then AUTO takes the 32-bit path
 * up to 2^24 points).  The plan is bound to the current CUDA device. */
int bw_plan_create(bw_plan** out, int path, size_t la, size_t lb,
                   int num_primes, unsigned flags);
int bw_plan_destroy(bw_plan* plan);
int bw_plan_get_info(const bw_plan* plan, bw_plan_info* out);

/* Allocate device scratch for one in-flight product of the plan's size.
 * stream = NULL creates a private non-blocking stream; otherwise work is
 * issued on the given cudaStream_t. */
int bw_ctx_create(bw_ctx** out, const bw_plan* plan, void* stream);
int bw_ctx_destroy(bw_ctx* ctx);

/* Host-pointer products (BW_PTR_HOST, BW_PTR_HOST_ASYNC) of large plans split
 * their copies into chunks that overlap the kernels at either end: the
 * copy-in goes in column blocks, and the first transform pass runs on each
 * block as soon as it has landed; the copy-out goes in word ranges, each
 * as soon as the carry pass has finished it.  The copies run on two more
 * streams of the context, and the context stream waits for them.
 * chunks = 0: automatic: whole copies while the plan has several live
 * contexts (their products already overlap one another's copies), else 8
 * from 2^23 product words, 4 from 2^21, 1 below; 1: whole copies on the
 * context stream; 2..16: that many (rounded down to a power of two and
 * capped by the plan's column tiles).  Calls with timing use whole
 * copies, so that the stage times stay separate.  Reference: the ingress
 * and egress of execute_ntt_multiply, src/gpu_ntt.cu:468-473,932-933. */
int bw_ctx_set_copy_chunks(bw_ctx* ctx, int chunks);
/* The cudaStream_t the context issues work on. */
void* bw_ctx_stream(const bw_ctx* ctx);
/* Wait for the context's stream and report device-side errors raised by
 * earlier BW_PTR_DEVICE calls (BW_ETIMEOUT, BW_ECHECK). */
int bw_ctx_sync(bw_ctx* ctx);

/* c[0 .. la+lb) = a[0 .. la) * b[0 .. lb).  lc must be >= la + lb; words of
 * c beyond la + lb are left untouched.  la and lb must equal the plan's.
 * a == b with la == lb multiplies a number by itself through the squaring
 * schedule (one forward transform).  timing may be NULL. */
int bw_multiply(bw_ctx* ctx, const uint32_t* a, size_t la,
                const uint32_t* b, size_t lb, uint32_t* c, size_t lc,
                unsigned flags, bw_timing* timing);

/* c = a * a with the squaring schedule. */
int bw_square(bw_ctx* ctx, const uint32_t* a, size_t la,
              uint32_t* c, size_t lc, unsigned flags, bw_timing* timing);

/* Stop after Garner: the n convolution coefficients of the product (in the
 * plan's coefficient base, 2^16 or 2^32) as three little-endian u32 words
 * each, words[3*i + w].  Host pointers only.  (Reference: the CRT dump of
 * execute_ntt_multiply, src/gpu_ntt.cu:843-884.) */
int bw_multiply_coeffs(bw_ctx* ctx, const uint32_t* a, size_t la,
                       const uint32_t* b, size_t lb, uint32_t* words,
                       size_t n_words);

/* Test hooks for the bounded device-side waits of the carry look-back.
 * bw_ctx_set_wait_limit sets how many polls (about 64 ns apart) a wait may
 * take before it gives up and the call reports BW_ETIMEOUT (default 2^22).
 * bw_ctx_inject_wait_fault(ctx, 1) makes the next products wait for a tile
 * flag that nothing sets, so every wait runs out; the context stays usable
 * and products are correct again after bw_ctx_inject_wait_fault(ctx, 0).
 * No counterpart in the reference (it checks no CUDA errors at all). */
int bw_ctx_set_wait_limit(bw_ctx* ctx, int polls);
int bw_ctx_inject_wait_fault(bw_ctx* ctx, int enable);

/* Largest number of 2048-word carry tiles bw_garner_carry_noalloc handles:
 * up to 2^26 output words (products of up to 2^31 bits). */
#define BW_NOALLOC_MAX_TILES 32768

/* Garner reconstruction + carry propagation of a finished cyclic
 * convolution, for callers that cannot allocate device memory.  Some host
 * programs give all device memory to their own pool allocator up front, so an
 * allocation inside a library fails or takes memory the pool counts on; others
 * cannot let a library call synchronise the whole device, which cudaFree does
 * (a serving loop that keeps other streams busy, for one).  This call
 * allocates nothing.  The caller passes residues (device memory, 16-byte
 * aligned): num_primes arrays of n fully reduced residues, array k at
 * residues + k * n elements, u64 elements for BW_PATH_P64 and u32 for
 * BW_PATH_P32, in natural coefficient order.  Accepted are the residues of
 * 32-bit coefficients on BW_PATH_P64 and of 16-bit coefficients on
 * BW_PATH_P32 (num_primes 2, or 3 with the third prime as a check; 0 means
 * 2), as plans with those coefficient widths leave them; residues of 64-bit
 * coefficients (BW_PLAN_COEF64) are not.  It writes out[0 .. min(out_words,
 * n / c + 1)) with c = 1 (P64) or 2 (P32: two 16-bit coefficients per word);
 * word n / c, when asked for, receives the final carry.  The primes are the
 * library's, see bw_plan_get_info.  n is a power of two >= 16 and the words
 * written fit BW_NOALLOC_MAX_TILES * 2048, else BW_ESIZE.  The look-back
 * scratch is one fixed-size device array in the library (about 640 KiB on
 * every GPU that loads it, kept until exit); every call shares it and clears
 * the part it uses, so calls whose GPU work overlaps (different streams or
 * threads) race: serialise them.  The call enqueues on `stream`, then reads
 * the device error word back and waits for the stream, so a stream that is
 * being captured is refused with BW_EINVAL before anything is enqueued.  The
 * first call on a device looks the array's device address up
 * (cudaGetSymbolAddress).  No counterpart in the reference: there, the CRT
 * and carry stages (src/crt_gpu.cu, src/carry_prop.cu) need buffers the
 * caller allocates with cudaMalloc. */
int bw_garner_carry_noalloc(int path, int num_primes, const void* residues, size_t n,
                            uint32_t* out, size_t out_words, void* stream);

/* Integer-pipe ceiling of the transforms: runs the library's own forward and
 * inverse butterflies of one prime path (BW_PATH_P32 or BW_PATH_P64) from
 * registers, with no memory traffic, on ctas_per_sm 256-thread CTAs per SM
 * of the current device, `iters` times 96 butterflies per thread.  Returns
 * the kernel's CUDA-event time and the butterflies it did; butterflies per
 * second divided by SMs and the SM clock is the per-SM-cycle ceiling that the
 * "fraction of the integer floor" figures divide by.  No counterpart in the
 * reference (its NTT is the absent GPU-NTT library). */
int bw_butterfly_rate(int path, int iters, int ctas_per_sm, float* ms,
                      double* butterflies);

/* One-shot convenience: plan + context + multiply, host pointers.
 * (Reference: host_multiply_merge, src/host_multiply.cpp:27-86, which
 * rebuilds its tables and context on every call.)  The plan and context of a
 * size stay cached for the next call of the same size, path and device, up
 * to bw_host_once_cache_limit bytes of device memory (least recently used
 * sizes are freed first; a size larger than the limit is freed after its
 * call).  Thread-safe: concurrent calls of one size use separate contexts. */
int bw_multiply_host_once(const uint32_t* a, size_t la, const uint32_t* b,
                          size_t lb, uint32_t* c, size_t lc, int path,
                          float* elapsed_ms);

/* Device memory the one-shot cache may hold (default 4 GiB); 0 frees every
 * idle entry and turns the cache off.  The cached plans and contexts belong
 * to the device's current CUDA context: call this with 0 before resetting
 * the device (cudaDeviceReset). */
int bw_host_once_cache_limit(size_t bytes);

/* ---------------------------------------------------------------- batches
 * Many independent products of uneven sizes in one launch sequence.  The
 * reference has no batched form (each product is one host_multiply_merge
 * call, src/host_multiply.cpp:27-86); these calls add it.
 *
 * Products are grouped by transform length; each group runs as one set of
 * kernels over all of its products (small groups: one CTA per whole
 * product; larger ones: the 4-step kernels with a product grid dimension).
 * The groups run concurrently inside one CUDA graph that is replayed for as
 * long as the list of products (their sizes) stays the same.  Transform
 * lengths up to 2^26 (P64: products of up to 2^26 words; P32: 2^25, within
 * the path's own limit). */
typedef struct bw_batch bw_batch;

#define BW_BATCH_THREE_PRIMES 1u  /* bw_batch_create: K = 3 (redundant check) */
/* bw_batch_create: the small buckets (one CTA per product) of each prime path
 * run as one persistent kernel that pulls (bucket, product) work items,
 * largest transforms first, from a device queue, instead of one grid per
 * bucket.  The other buckets are unchanged.  A measured alternative to the
 * default graph of per-bucket grids. */
#define BW_BATCH_PERSISTENT 2u

/* bw_batch_run `what` bits (0 = all three) */
#define BW_BATCH_UPLOAD 1u    /* copy every product's operands to the device */
#define BW_BATCH_COMPUTE 2u   /* run the products */
#define BW_BATCH_DOWNLOAD 4u  /* copy every result back to its host buffer */

typedef struct {
    size_t products;
    size_t buckets;        /* groups of equal transform length */
    size_t small_buckets;  /* groups run one CTA per product */
    size_t graph_nodes;    /* nodes of the captured graph */
    size_t device_bytes;   /* device memory the batch holds */
    size_t kernel_nodes;   /* kernel launches per run (the graph's kernel nodes) */
} bw_batch_info;

/* stream = NULL creates a private stream. */
int bw_batch_create(bw_batch** out, void* stream, unsigned flags);
int bw_batch_destroy(bw_batch* batch);
/* Forget every product (the device buffers are kept for reuse). */
int bw_batch_clear(bw_batch* batch);
/* Append c[0 .. la+lb) = a * b (host pointers, read at every run with
 * BW_BATCH_UPLOAD; c written at every run with BW_BATCH_DOWNLOAD).
 * a == b with la == lb squares.  path BW_PATH_AUTO chooses as
 * bw_plan_create does. */
int bw_batch_add(bw_batch* batch, int path, const uint32_t* a, size_t la,
                 const uint32_t* b, size_t lb, uint32_t* c, size_t lc);
/* Run the batch (blocking).  The first run after bw_batch_add/clear builds
 * the groups and captures the graph.  timing gets h2d_ms, mul_ms, d2h_ms and
 * total_ms.  BW_ECHECK / BW_ETIMEOUT as for bw_multiply. */
int bw_batch_run(bw_batch* batch, unsigned what, bw_timing* timing);
int bw_batch_get_info(const bw_batch* batch, bw_batch_info* info);
/* Test hooks for the bounded look-back waits of the 4-step groups, as for
 * contexts (bw_ctx_set_wait_limit / bw_ctx_inject_wait_fault): a run with the
 * fault injected reports BW_ETIMEOUT, and the batch is correct again once
 * it is switched off.  Both rebuild the captured graph at the next run. */
int bw_batch_set_wait_limit(bw_batch* batch, int polls);
int bw_batch_inject_wait_fault(bw_batch* batch, int enable);

/* Time each candidate form of each group (one CTA per product where the
 * transform fits shared memory; 4-step with each column/row split from
 * square to long rows, each with row rounds of radix 8 and 16) on the
 * batch's own products, `reps` runs each, and keep the fastest in the
 * process-wide tune table that later layouts use.  Blocking. */
int bw_batch_autotune(bw_batch* batch, int reps);
/* The tune table as a JSON array of {path, num_primes, log_n, small,
 * log_cols, row_radix, ms}.  Writes at most len bytes including the
 * terminating NUL; *needed gets the full size. */
int bw_tune_table_export(char* buf, size_t len, size_t* needed);
/* Set one tune-table entry (log_cols 0 = automatic split; row_radix 8 or 16,
 * or 0 for the path's default: 8 on the 64-bit path, 16 on the 32-bit). */
int bw_tune_table_set(int path, int num_primes, int log_n, int small, int log_cols,
                      int row_radix);

/* ---------------------------------------------------------------- serving
 * A request loop with continuous batching.  Requests (host buffers) are
 * submitted from any thread as they arrive and finish asynchronously.  Two
 * library threads run the loop: one admits waiting requests in arrival
 * order while the device bytes they need fit the budget, groups them by
 * transform length and issues each group as one batched launch on one of
 * several streams (at most max_groups_in_flight groups on the device; what
 * arrives meanwhile is admitted together into the next groups); the other
 * detects finished groups, copies results out and frees their memory.
 * Twiddle tables stay resident between requests.  No reference counterpart:
 * the reference multiplies one product per blocking host_multiply_merge call
 * (src/host_multiply.cpp:27-86). */
typedef struct bw_server bw_server;

typedef struct bw_server_config {
    size_t   hbm_budget_bytes;      /* admission budget: resident tables +
                                       in-flight groups (0 = 120 GiB)       */
    size_t   pinned_bytes;          /* host staging (0 = 2 GiB)             */
    int      lanes;                 /* streams groups are issued on (0 = 8) */
    int      max_groups_in_flight;  /* (0 = 2 * lanes)                      */
    int      num_primes;            /* K (0 = 2)                            */
    int      path;                  /* default path (BW_PATH_AUTO: chosen
                                       per request, as for bw_plan_create)  */
} bw_server_config;

/* One finished request.  Times are microseconds on a steady clock since the
 * server was created; admit/launch are -1 for a request that never ran. */
typedef struct bw_request_info {
    uint64_t ticket;
    int      status;        /* BW_OK, or why the request failed            */
    double   submit_us, admit_us, launch_us, done_us;
    size_t   group_size;    /* products in the launch group it ran in      */
    size_t   device_bytes;  /* bytes charged against the budget            */
    size_t   la, lb;
} bw_request_info;

typedef struct bw_server_stats {
    uint64_t submitted, completed, rejected, failed;
    uint64_t groups, kernel_launches;
    size_t   max_group_size;
    size_t   bytes_in_flight, peak_bytes_in_flight;  /* incl. resident tables */
    size_t   resident_plan_bytes, queue_depth, groups_in_flight, budget_bytes;
} bw_server_stats;

/* cfg may be NULL (all defaults).  Uses the current CUDA device. */
int bw_server_create(bw_server** out, const bw_server_config* cfg);
/* Waiting requests fail with BW_EBUSY; admitted ones finish first. */
int bw_server_destroy(bw_server* server);
/* Build the resident tables for every transform length up to 2^max_log_n. */
int bw_server_prewarm(bw_server* server, int path, int max_log_n);
/* Queue c[0 .. la+lb) = a * b.  a, b and c must stay valid until the
 * request finishes.  a == b with la == lb squares.  BW_EREJECT when the
 * request alone needs more than the budget; BW_ESIZE beyond the limits
 * (transform length 2^26 at most). */
int bw_server_submit(bw_server* server, int path, const uint32_t* a, size_t la,
                     const uint32_t* b, size_t lb, uint32_t* c, size_t lc,
                     uint64_t* ticket);
/* Wait for one request (timeout_ms < 0: no limit; 0: poll) and release it.
 * Returns its status, or BW_ETIMEOUT if it has not finished. */
int bw_server_wait(bw_server* server, uint64_t ticket, int timeout_ms,
                   bw_request_info* info);
/* Take up to max finished requests (any order) and release them. */
int bw_server_harvest(bw_server* server, bw_request_info* out, size_t max,
                      size_t* count);
/* Wait until nothing is waiting or running. */
int bw_server_drain(bw_server* server, int timeout_ms);
int bw_server_get_stats(bw_server* server, bw_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* BIRDWING_H */
