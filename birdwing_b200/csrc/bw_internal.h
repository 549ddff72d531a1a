// bw_internal.h -- plan layout shared by the library's translation units.
#pragma once
#include <cstddef>
#include <cstdint>
#include <mutex>

#include "bw_kernels.cuh"

// Stage order of the host-pointer products of one plan.  Contexts of one
// plan used in turn form a three-stage pipeline (copy-in, kernels,
// copy-out): each stage of a product waits for the same stage of the plan's
// previous product, so every stage runs alone at full speed while the three
// overlap.  Unordered, the products in flight share the PCIe link and the SMs
// evenly and finish together, and the copies hide little of the kernels.
// Only plans with more than one live context order their products.
struct bw_stage_order {
    std::mutex mu;
    int contexts = 0;              // live contexts of the plan
    cudaEvent_t last[3] = {};      // end of the previous product's stage i
    const void* owner[3] = {};     // context that recorded last[i]
};

struct bw_plan {
    int path = 0, K = 0;
    size_t la = 0, lb = 0, nca = 0, ncb = 0;
    int log_n = 0, log_r = 0, log_c = 0, log_cb = 0, lo = 0;
    int log_cb1 = 0;     // forward column pass tile width (its own shared-memory budget)
    int tw_smem_r = 0;   // column stage twiddles staged in shared memory
    int rlog_row = 4;    // radix of the row kernel's rounds (2^3 or 2^4)
    int rlog_col = 4;    // radix of the column kernels' rounds (single products, 64-bit path)
    int log_r2 = 0;      // three-pass schedule: middle column length (0: two passes)
    int log_cb2 = 0, lo_out = 0;
    int small = 0;       // single-pass plan: the whole n-point transform in one CTA
    int w64 = 0;         // 64-bit coefficients (two words each): K = 3 on the 64-bit
                         // path, K = 6 on the 32-bit path
    int tma_cols = 0;    // inverse column tiles by tensor copies (BW_PLAN_TMA_COLS)
    int shfl_rows = 0;   // row pass exchange through warp shuffles (BW_PLAN_SHFL_ROWS)
    int k1_pp = 0;       // 32-bit path, 64-bit coefficients: one prime per forward-pass CTA
    int coef_half = 0;   // ... prime loop: both operands in the low half, half the u64 copy
    int device = 0;
    bool zt_a = false, zt_b = false;
    void* d_tables = nullptr;
    size_t table_bytes = 0;
    bw::PlanDev<bw::Ar32> pd32{};
    bw::PlanDev<bw::Ar64> pd64{};
    uint64_t primes[bw::kMaxPrimes] = {};
    bw_stage_order* order = nullptr;  // plans of bw_plan_create only
};

// Split, tables and constants of a plan for transform length 2^log_n.
// mode 0: the 4-step pipeline (two or three passes) for batch groups;
// mode 1: single-pass products of one CTA each (n-point stage tables and the
// n^-1 scale); mode 2: the 4-step pipeline for one product at a time, with
// column tiles narrowed for small n so that the column passes fill the SMs.
int bw_plan_setup(bw_plan* pl, int path, int K, int log_n, unsigned flags, int mode);

// Set the dynamic shared-memory limit of every kernel instantiation once.
int bw_set_kernel_attrs();

// Largest transform of a launch group: the two-pass schedule.
constexpr int kMaxGroupLogN = 26;

// One launch group: np products of one plan (equal path, K and transform
// length), product q described by d_desc[q].  A single-pass plan (small)
// runs ks_product, one CTA per product, with residue scratch res_a
// (np * K * n elements); a 4-step plan runs kb_fwd_col, kb_row, kb_inv_col
// and kb_garner_carry over residue arenas res_a and res_b of the same size,
// with per-product look-back state (zeroed before the launch, epoch 1).
struct bw_group_launch {
    const bw_plan* plan;
    const bw::BatchProd* d_desc;
    unsigned np;
    void* res_a;
    void* res_b;
    size_t ntiles;      // carry tiles per product (bw_group_ntiles)
    uint32_t* d_err;    // bit 0: look-back wait timed out; bit 1: check failed
    int spin_limit;
    bool inject_wait_fault = false;  // test hook: every look-back wait runs out
    int rlog = 0;       // row-pass radix log2 (0: radix 8 on the 64-bit path, 16 on the 32-bit)
};
int bw_enqueue_group(const bw_group_launch& g, cudaStream_t s);
// Carry tiles of a group whose longest product has max_words output words.
size_t bw_group_ntiles(int path, int log_n, size_t max_words);
// Bytes of one product's look-back state (16-byte multiple).
size_t bw_group_state_stride(size_t ntiles);
// Kernel form (single-pass or 4-step) and 4-step split for a transform
// length, from the tune table (bw_batch_autotune / bw_tune_table_set).
void bw_tune_lookup(int path, int K, int log_n, int* small, int* log_cols);
// Point a descriptor's look-back fields into its state block.
void bw_group_fill_state(bw::BatchProd& d, unsigned char* state, size_t ntiles);
