// bw_batch.cu -- many products of uneven sizes per launch (bw_batch_* in
// birdwing.h).
//
// Products are grouped into buckets of equal (prime path, K, transform
// length).  A bucket runs as one set of kernels over all of its products:
//   small buckets  ks_product: one CTA per whole product (transforms,
//                  product, inverse, Garner and carry in shared memory);
//   larger buckets the 4-step kernels with a product grid dimension
//                  (kb_fwd_col, kb_row, kb_inv_col, kb_garner_carry), each
//                  product reading its own descriptor.
// All buckets are captured in one CUDA graph whose branches run on separate
// streams; the graph is replayed while the batch's size layout does not
// change.  Per bucket the kernel form (small or 4-step) and the 4-step split
// come from a tune table that bw_batch_autotune fills by timing the
// candidates on the batch's own products; the table can be exported and
// imported as JSON.
//
// The reference has no batched form: each product is one call of
// host_multiply_merge (src/host_multiply.cpp:27-86).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/birdwing.h"
#include "bw_host.h"
#include "bw_internal.h"
#include "bw_kernels.cuh"

using namespace bw;

namespace {

#define BW_TRY(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return bw_fail(e_ == cudaErrorMemoryAllocation ? BW_ENOMEM : BW_ECUDA,        \
                           "%s failed: %s", #call, cudaGetErrorString(e_));               \
    } while (0)

// ---- tune table: (path, K, log_n) -> kernel form, split and row radix
struct TuneKey {
    int path, K, log_n;
    bool operator<(const TuneKey& o) const {
        return std::tie(path, K, log_n) < std::tie(o.path, o.K, o.log_n);
    }
};
struct TuneVal {
    int small;     // 1: one CTA per product
    int log_cols;  // 4-step split (0 = automatic)
    int rlog;      // row-pass radix log2, 3 or 4 (0 = the path's default)
    float ms;      // measured time of the bucket when tuned (0 = default)
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune;

// The one-CTA kernel holds both operands' transforms in shared memory: up to
// 2^13 (64-bit) or 2^14 (32-bit) points.  By default it runs up to 2^12
// points; beyond that the 4-step kernels measured faster on both paths (the
// one-CTA kernel's shared memory then holds one or two CTAs per SM).
int small_max_log(int path) { return path == BW_PATH_P64 ? 13 : 14; }
constexpr int kSmallDefaultLog = 12;

// Products per bucket: kb_fwd_col puts 2 * products in gridDim.z (<= 65535).
constexpr size_t kMaxBucket = 16384;

// Threads of the persistent small-product kernel (BW_BATCH_PERSISTENT).
constexpr int kQueueThreads = 256;

TuneVal tune_get(int path, int K, int log_n) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(TuneKey{path, K, log_n});
    if (it != g_tune.end()) return it->second;
    return TuneVal{log_n <= kSmallDefaultLog ? 1 : 0, 0, 0, 0.f};
}

struct Prod {
    int path = 0;
    const uint32_t* a = nullptr;
    const uint32_t* b = nullptr;
    uint32_t* c = nullptr;
    size_t la = 0, lb = 0, lc = 0;
    bool square = false;
    int log_n = 0;
    size_t in_a = 0, in_b = 0, out = 0;  // word offsets in the staging arenas
};

struct Bucket {
    int path = 0, K = 2, log_n = 0;
    int small = 0, log_cols = 0, rlog = 0;
    bw_plan plan;
    std::vector<size_t> prods;
    BatchProd* d_desc = nullptr;
    void* d_res_a = nullptr;
    void* d_res_b = nullptr;
    unsigned char* d_state = nullptr;
    size_t ntiles = 0;
};

// Host staging copies of a batch (operands into pinned memory, results out of
// it) split over a few threads: one thread's memcpy bandwidth bounded the
// batch's end-to-end rate.
template <class F>
void parallel_products(size_t lo, size_t hi, size_t bytes, F fn) {
    const size_t count = hi - lo;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>({8, hw, std::max<size_t>(1, bytes >> 22), count});
    if (nt <= 1) {
        for (size_t i = lo; i < hi; ++i) fn(i);
        return;
    }
    std::vector<std::thread> th;
    for (size_t t = 0; t < nt; ++t)
        th.emplace_back([&, t] {
            for (size_t i = lo + t * count / nt; i < lo + (t + 1) * count / nt; ++i) fn(i);
        });
    for (auto& x : th) x.join();
}

// The staging copies and the DMA overlap chunk by chunk.
constexpr size_t kStageChunks = 4;

void free_bucket(Bucket& b) {
    cudaFree(b.d_desc);
    cudaFree(b.d_res_a);
    cudaFree(b.d_res_b);
    cudaFree(b.d_state);
    cudaFree(b.plan.d_tables);
    b.d_desc = nullptr;
    b.d_res_a = b.d_res_b = nullptr;
    b.d_state = nullptr;
    b.plan.d_tables = nullptr;
}

}  // namespace

struct bw_batch {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int K = 2;
    std::vector<Prod> prods;
    std::vector<Bucket> buckets;
    bool dirty = true;
    uint32_t* d_in = nullptr;
    uint32_t* d_out = nullptr;
    uint32_t* h_in = nullptr;   // pinned staging
    uint32_t* h_out = nullptr;  // pinned staging
    size_t in_words = 0, out_words = 0, in_cap = 0, out_cap = 0;
    uint32_t* d_err = nullptr;
    uint32_t* h_err = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    static constexpr int kSide = 8;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork = nullptr, join[kSide] = {};
    cudaEvent_t ev[4] = {};
    cudaEvent_t chunk_ev[kStageChunks] = {};
    size_t graph_nodes = 0;
    size_t kernel_nodes = 0;
    int spin_limit = 1 << 22;
    bool inject_wait_fault = false;
    // BW_BATCH_PERSISTENT: per prime path (0: 64-bit, 1: 32-bit), the small
    // buckets' device table, their work items and the queue head
    bool persistent = false;
    void* d_qbuckets[2] = {};
    SmallItem* d_qitems[2] = {};
    uint32_t* d_qhead = nullptr;  // two counters
    uint32_t qcount[2] = {0, 0};
    int qlog_max[2] = {0, 0};
};

namespace {

void drop_queues(bw_batch* bt) {
    for (int i = 0; i < 2; ++i) {
        cudaFree(bt->d_qbuckets[i]);
        cudaFree(bt->d_qitems[i]);
        bt->d_qbuckets[i] = nullptr;
        bt->d_qitems[i] = nullptr;
        bt->qcount[i] = 0;
        bt->qlog_max[i] = 0;
    }
}

void drop_layout(bw_batch* bt) {
    drop_queues(bt);
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    bt->exec = nullptr;
    bt->graph = nullptr;
    for (auto& b : bt->buckets) free_bucket(b);
    bt->buckets.clear();
}

}  // namespace

// ---- launch groups (shared with the serving engine)
namespace {

template <class Ar>
const PlanDev<Ar>& pdev(const bw_plan& p);
template <>
const PlanDev<Ar32>& pdev<Ar32>(const bw_plan& p) {
    return p.pd32;
}
template <>
const PlanDev<Ar64>& pdev<Ar64>(const bw_plan& p) {
    return p.pd64;
}

template <class Ar, bool SPLIT16>
void enqueue_group_t(const bw_group_launch& g, cudaStream_t s) {
    using T = typename Ar::T;
    const bw_plan& pl = *g.plan;
    const PlanDev<Ar>& P = pdev<Ar>(pl);
    const unsigned np = g.np;
    T* ra = static_cast<T*>(g.res_a);
    T* rb = static_cast<T*>(g.res_b);
    if (pl.small) {
        const int n = 1 << pl.log_n;
        const size_t smem = 2 * tile_elems(n) * sizeof(T);
        const int want = std::min(256, std::max(64, n >> 4));
        if (want >= 256) {
            ks_product<Ar, SPLIT16, 256><<<np, 256, smem, s>>>(P, g.d_desc, ra, g.d_err);
        } else if (want >= 128) {
            ks_product<Ar, SPLIT16, 128><<<np, 128, smem, s>>>(P, g.d_desc, ra, g.d_err);
        } else {
            ks_product<Ar, SPLIT16, 64><<<np, 64, smem, s>>>(P, g.d_desc, ra, g.d_err);
        }
        return;
    }
    const int R = 1 << pl.log_r, C = 1 << pl.log_c, CB = 1 << pl.log_cb;
    const int CB1 = 1 << pl.log_cb1;
    const size_t smem1 = tile_elems((size_t)R * CB1) * sizeof(T) + (size_t)R * CB1 * (SPLIT16 ? 2 : 4);
    kb_fwd_col<Ar, SPLIT16, 4><<<dim3(C / CB1, 1, 2 * np), kColThreads, smem1, s>>>(
        P, g.d_desc, ra, rb);
    const int la = pl.log_c / 2;
    const size_t ntab = 2 * (((size_t)1 << la) + ((size_t)C >> la));
    const size_t smem2 = ntab * sizeof(Tw<T>) + tile_elems(C) * sizeof(T) * 2;
    const dim3 g2(R, pl.K, np);
    // row rounds: radix 8 on the 64-bit path (at most 256 threads, 64
    // registers, as its single-product row pass), radix 16 on the 32-bit
    // path, unless the tune table chose the other radix for the bucket
    const int rl = g.rlog ? g.rlog : (sizeof(T) == 8 ? 3 : 4);
    if (rl == 3) {
        switch (std::min(sizeof(T) == 8 ? 256 : 512, std::max(64, C >> 3))) {
            case 512: kb_row<Ar, 512, 3><<<g2, 512, smem2, s>>>(P, g.d_desc, ra, rb); break;
            case 256: kb_row<Ar, 256, 3><<<g2, 256, smem2, s>>>(P, g.d_desc, ra, rb); break;
            case 128: kb_row<Ar, 128, 3><<<g2, 128, smem2, s>>>(P, g.d_desc, ra, rb); break;
            default: kb_row<Ar, 64, 3><<<g2, 64, smem2, s>>>(P, g.d_desc, ra, rb); break;
        }
    } else {
        switch (std::min(512, std::max(64, C >> 4))) {
            case 512: kb_row<Ar, 512, 4><<<g2, 512, smem2, s>>>(P, g.d_desc, ra, rb); break;
            case 256: kb_row<Ar, 256, 4><<<g2, 256, smem2, s>>>(P, g.d_desc, ra, rb); break;
            case 128: kb_row<Ar, 128, 4><<<g2, 128, smem2, s>>>(P, g.d_desc, ra, rb); break;
            default: kb_row<Ar, 64, 4><<<g2, 64, smem2, s>>>(P, g.d_desc, ra, rb); break;
        }
    }
    const size_t smem3 = tile_elems((size_t)R * CB) * sizeof(T);
    kb_inv_col<Ar, 4><<<dim3(C / CB, pl.K, np), kColThreads, smem3, s>>>(P, g.d_desc, ra);
    kb_garner_carry<Ar, SPLIT16><<<dim3((unsigned)g.ntiles, np), kCarryThreads, 0, s>>>(
        P, g.d_desc, ra, 1u, g.inject_wait_fault ? 1u + (1u << 27) : 1u, g.d_err, g.spin_limit);
}

int set_group_attrs() {
    static std::once_flag once;
    static cudaError_t st = cudaSuccess;
    std::call_once(once, [] {
        auto set = [](const void* f) {
            cudaError_t e =
                cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if (e != cudaSuccess) st = e;
        };
        set((const void*)ks_product<Ar64, false, 64>);
        set((const void*)ks_product<Ar64, false, 128>);
        set((const void*)ks_product<Ar64, false, 256>);
        set((const void*)ks_product<Ar32, true, 64>);
        set((const void*)ks_product<Ar32, true, 128>);
        set((const void*)ks_product<Ar32, true, 256>);
        set((const void*)kq_small<Ar64, false, kQueueThreads>);
        set((const void*)kq_small<Ar32, true, kQueueThreads>);
        set((const void*)kb_fwd_col<Ar64, false, 4>);
        set((const void*)kb_fwd_col<Ar32, true, 4>);
        set((const void*)kb_inv_col<Ar64, 4>);
        set((const void*)kb_inv_col<Ar32, 4>);
        for (auto f : {(const void*)kb_row<Ar64, 64, 3>, (const void*)kb_row<Ar64, 128, 3>,
                       (const void*)kb_row<Ar64, 256, 3>, (const void*)kb_row<Ar64, 512, 3>,
                       (const void*)kb_row<Ar64, 64, 4>, (const void*)kb_row<Ar64, 128, 4>,
                       (const void*)kb_row<Ar64, 256, 4>, (const void*)kb_row<Ar64, 512, 4>,
                       (const void*)kb_row<Ar32, 64, 3>, (const void*)kb_row<Ar32, 128, 3>,
                       (const void*)kb_row<Ar32, 256, 3>, (const void*)kb_row<Ar32, 512, 3>,
                       (const void*)kb_row<Ar32, 64, 4>, (const void*)kb_row<Ar32, 128, 4>,
                       (const void*)kb_row<Ar32, 256, 4>, (const void*)kb_row<Ar32, 512, 4>})
            set(f);
    });
    if (st != cudaSuccess)
        return bw_fail(BW_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(st));
    return BW_OK;
}

}  // namespace

int bw_enqueue_group(const bw_group_launch& g, cudaStream_t s) {
    int rc = set_group_attrs();
    if (rc) return rc;
    if (g.plan->path == BW_PATH_P64) {
        enqueue_group_t<Ar64, false>(g, s);
    } else {
        enqueue_group_t<Ar32, true>(g, s);
    }
    return BW_OK;
}

size_t bw_group_ntiles(int path, int log_n, size_t max_words) {
    const size_t NL = ((size_t)1 << log_n) / (path == BW_PATH_P32 ? 2 : 1);
    const size_t words = std::max(NL, max_words);
    return (words + kCarryTileWords - 1) / kCarryTileWords;
}

void bw_tune_lookup(int path, int K, int log_n, int* small, int* log_cols) {
    const TuneVal tv = tune_get(path, K, log_n);
    *small = tv.small && log_n <= small_max_log(path);
    *log_cols = tv.log_cols;
}

size_t bw_group_state_stride(size_t ntiles) { return ((16 + ntiles * 20) + 15) & ~(size_t)15; }

void bw_group_fill_state(bw::BatchProd& d, unsigned char* state, size_t ntiles) {
    d.cst = reinterpret_cast<CarryState*>(state);
    d.rec_x = reinterpret_cast<uint4*>(state + 16);
    d.rec_s = reinterpret_cast<uint32_t*>(state + 16 + ntiles * 16);
}

namespace {

// BW_BATCH_PERSISTENT: the device table of one path's small buckets and its
// work items, largest transforms first.
template <class Ar>
int upload_queue(bw_batch* bt, int slot, const std::vector<size_t>& sb) {
    std::vector<SmallBucketDev<Ar>> tab(sb.size());
    std::vector<SmallItem> items;
    int log_max = 0;
    for (size_t j = 0; j < sb.size(); ++j) {
        const Bucket& bk = bt->buckets[sb[j]];
        tab[j].plan = pdev<Ar>(bk.plan);
        tab[j].desc = bk.d_desc;
        tab[j].scratch = static_cast<typename Ar::T*>(bk.d_res_a);
        log_max = std::max(log_max, bk.log_n);
        for (size_t q = 0; q < bk.prods.size(); ++q)
            items.push_back(SmallItem{(uint32_t)j, (uint32_t)q});
    }
    std::stable_sort(items.begin(), items.end(), [&](const SmallItem& x, const SmallItem& y) {
        return bt->buckets[sb[x.bucket]].log_n > bt->buckets[sb[y.bucket]].log_n;
    });
    BW_TRY(cudaMalloc(&bt->d_qbuckets[slot], tab.size() * sizeof(SmallBucketDev<Ar>)));
    BW_TRY(cudaMemcpy(bt->d_qbuckets[slot], tab.data(), tab.size() * sizeof(SmallBucketDev<Ar>),
                      cudaMemcpyHostToDevice));
    BW_TRY(cudaMalloc(&bt->d_qitems[slot], items.size() * sizeof(SmallItem)));
    BW_TRY(cudaMemcpy(bt->d_qitems[slot], items.data(), items.size() * sizeof(SmallItem),
                      cudaMemcpyHostToDevice));
    bt->qcount[slot] = (uint32_t)items.size();
    bt->qlog_max[slot] = log_max;
    return BW_OK;
}

// One path's queue kernel: as many CTAs as fit on the SMs at the largest
// transform's shared memory.
template <class Ar, bool SPLIT16>
cudaError_t launch_queue(bw_batch* bt, int slot, cudaStream_t s) {
    using T = typename Ar::T;
    const size_t smem = 2 * tile_elems((size_t)1 << bt->qlog_max[slot]) * sizeof(T);
    auto kern = kq_small<Ar, SPLIT16, kQueueThreads>;
    int per_sm = 0, dev = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kQueueThreads, smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const unsigned grid = (unsigned)std::min<size_t>((size_t)std::max(per_sm, 1) * sms,
                                                     bt->qcount[slot]);
    kern<<<grid, kQueueThreads, smem, s>>>(
        static_cast<const SmallBucketDev<Ar>*>(bt->d_qbuckets[slot]), bt->d_qitems[slot],
        bt->qcount[slot], bt->d_qhead + slot, bt->d_err);
    return cudaGetLastError();
}

// Build (or rebuild) buckets, arenas, descriptors and the graph.
int build_layout(bw_batch* bt) {
    drop_layout(bt);
    int rc = BW_OK;
    // staging offsets (16-byte aligned) and buckets
    std::map<std::tuple<int, int, int>, size_t> index;
    size_t in_w = 0, out_w = 0;
    auto align4 = [](size_t x) { return (x + 3) & ~(size_t)3; };
    for (size_t i = 0; i < bt->prods.size(); ++i) {
        Prod& p = bt->prods[i];
        p.in_a = in_w;
        in_w += align4(p.la);
        if (!p.square) {
            p.in_b = in_w;
            in_w += align4(p.lb);
        } else {
            p.in_b = p.in_a;
        }
        p.out = out_w;
        out_w += align4(p.la + p.lb);
        const auto key = std::make_tuple(p.path, bt->K, p.log_n);
        auto it = index.find(key);
        // a bucket holds at most kMaxBucket products (grid-dimension limits)
        if (it != index.end() && bt->buckets[it->second].prods.size() >= kMaxBucket) {
            index.erase(it);
            it = index.end();
        }
        if (it == index.end()) {
            Bucket b;
            b.path = p.path;
            b.K = bt->K;
            b.log_n = p.log_n;
            const TuneVal tv = tune_get(p.path, bt->K, p.log_n);
            b.small = tv.small && p.log_n <= small_max_log(p.path);
            b.log_cols = tv.log_cols;
            b.rlog = tv.rlog;
            index[key] = bt->buckets.size();
            bt->buckets.push_back(std::move(b));
            it = index.find(key);
        }
        bt->buckets[it->second].prods.push_back(i);
    }
    // arenas
    if (in_w > bt->in_cap) {
        cudaFree(bt->d_in);
        cudaFreeHost(bt->h_in);
        bt->d_in = nullptr;
        bt->h_in = nullptr;
        BW_TRY(cudaMalloc(&bt->d_in, std::max<size_t>(in_w, 4) * 4));
        BW_TRY(cudaMallocHost(&bt->h_in, std::max<size_t>(in_w, 4) * 4));
        bt->in_cap = in_w;
    }
    if (out_w > bt->out_cap) {
        cudaFree(bt->d_out);
        cudaFreeHost(bt->h_out);
        bt->d_out = nullptr;
        bt->h_out = nullptr;
        BW_TRY(cudaMalloc(&bt->d_out, std::max<size_t>(out_w, 4) * 4));
        BW_TRY(cudaMallocHost(&bt->h_out, std::max<size_t>(out_w, 4) * 4));
        bt->out_cap = out_w;
    }
    bt->in_words = in_w;
    bt->out_words = out_w;
    // per bucket: plan, residues, carry state, descriptors
    for (Bucket& bk : bt->buckets) {
        const unsigned flags = BW_PLAN_LOG_COLS(bk.log_cols);
        rc = bw_plan_setup(&bk.plan, bk.path, bk.K, bk.log_n, flags, bk.small ? 1 : 0);
        if (rc) return rc;
        const size_t n = (size_t)1 << bk.log_n;
        const int w = bk.path == BW_PATH_P64 ? 8 : 4;
        const int cpw = bk.path == BW_PATH_P32 ? 2 : 1;
        const size_t np = bk.prods.size();
        const size_t per = (size_t)bk.K * n;
        BW_TRY(cudaMalloc(&bk.d_res_a, np * per * w));
        if (!bk.small) BW_TRY(cudaMalloc(&bk.d_res_b, np * per * w));
        size_t maxw = n / cpw;
        for (size_t i : bk.prods) maxw = std::max(maxw, bt->prods[i].la + bt->prods[i].lb);
        bk.ntiles = bw_group_ntiles(bk.path, bk.log_n, maxw);
        const size_t st_stride = bw_group_state_stride(bk.ntiles);
        if (!bk.small) BW_TRY(cudaMalloc(&bk.d_state, np * st_stride));
        std::vector<BatchProd> desc(np);
        for (size_t q = 0; q < np; ++q) {
            const Prod& p = bt->prods[bk.prods[q]];
            BatchProd& d = desc[q];
            d.a = bt->d_in + p.in_a;
            d.b = bt->d_in + p.in_b;
            d.out = bt->d_out + p.out;
            d.la = (uint32_t)p.la;
            d.lb = (uint32_t)p.lb;
            d.square = p.square ? 1u : 0u;
            d.pad = 0;
            d.res_off = q * per;
            if (!bk.small) {
                bw_group_fill_state(d, bk.d_state + q * st_stride, bk.ntiles);
            } else {
                d.cst = nullptr;
                d.rec_x = nullptr;
                d.rec_s = nullptr;
            }
        }
        BW_TRY(cudaMalloc(&bk.d_desc, np * sizeof(BatchProd)));
        BW_TRY(cudaMemcpy(bk.d_desc, desc.data(), np * sizeof(BatchProd), cudaMemcpyHostToDevice));
    }
    // persistent form: one work queue per path over its small buckets
    if (bt->persistent) {
        if (!bt->d_qhead) BW_TRY(cudaMalloc(&bt->d_qhead, 2 * sizeof(uint32_t)));
        for (int slot = 0; slot < 2; ++slot) {
            const int path = slot == 0 ? BW_PATH_P64 : BW_PATH_P32;
            std::vector<size_t> sb;
            for (size_t i = 0; i < bt->buckets.size(); ++i)
                if (bt->buckets[i].small && bt->buckets[i].path == path) sb.push_back(i);
            if (sb.empty()) continue;
            rc = slot == 0 ? upload_queue<Ar64>(bt, slot, sb) : upload_queue<Ar32>(bt, slot, sb);
            if (rc) return rc;
        }
    }
    // graph: clear look-back state and the error word, then every bucket on
    // its own branch
    BW_TRY(cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    auto chk = [&](cudaError_t e) {
        if (ce == cudaSuccess) ce = e;
    };
    chk(cudaMemsetAsync(bt->d_err, 0, 4, bt->stream));
    if (bt->persistent) chk(cudaMemsetAsync(bt->d_qhead, 0, 2 * sizeof(uint32_t), bt->stream));
    for (const Bucket& bk : bt->buckets) {
        if (bk.d_state) {
            chk(cudaMemsetAsync(bk.d_state, 0, bk.prods.size() * bw_group_state_stride(bk.ntiles),
                                bt->stream));
        }
    }
    chk(cudaEventRecord(bt->fork, bt->stream));
    const int nside = (int)std::min<size_t>(bw_batch::kSide, bt->buckets.size());
    for (int s = 0; s < nside; ++s) chk(cudaStreamWaitEvent(bt->side[s], bt->fork, 0));
    // largest buckets first, round-robin over the branches
    std::vector<size_t> order(bt->buckets.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t x, size_t y) {
        const auto& a = bt->buckets[x];
        const auto& b = bt->buckets[y];
        return (a.prods.size() << a.log_n) > (b.prods.size() << b.log_n);
    });
    // the persistent queues first (one branch per path), then the other
    // buckets round-robin after them
    size_t branch = 0;
    if (bt->persistent) {
        rc = set_group_attrs();
        for (int slot = 0; slot < 2 && rc == BW_OK; ++slot) {
            if (!bt->qcount[slot]) continue;
            chk(slot == 0 ? launch_queue<Ar64, false>(bt, slot, bt->side[branch % nside])
                          : launch_queue<Ar32, true>(bt, slot, bt->side[branch % nside]));
            ++branch;
        }
    }
    for (size_t i = 0; i < order.size() && rc == BW_OK; ++i) {
        const Bucket& bk = bt->buckets[order[i]];
        if (bt->persistent && bk.small) continue;
        bw_group_launch g{&bk.plan, bk.d_desc, (unsigned)bk.prods.size(), bk.d_res_a,
                          bk.d_res_b, bk.ntiles, bt->d_err, bt->spin_limit,
                          bt->inject_wait_fault, bk.rlog};
        rc = bw_enqueue_group(g, bt->side[branch++ % nside]);
    }
    for (int s = 0; s < nside; ++s) {
        chk(cudaEventRecord(bt->join[s], bt->side[s]));
        chk(cudaStreamWaitEvent(bt->stream, bt->join[s], 0));
    }
    chk(cudaGetLastError());
    cudaError_t e = cudaStreamEndCapture(bt->stream, &bt->graph);
    if (rc) return rc;
    if (ce != cudaSuccess) return bw_fail(BW_ECUDA, "batch capture: %s", cudaGetErrorString(ce));
    if (e != cudaSuccess) return bw_fail(BW_ECUDA, "end capture: %s", cudaGetErrorString(e));
    BW_TRY(cudaGraphInstantiate(&bt->exec, bt->graph, 0));
    size_t nodes = 0;
    cudaGraphGetNodes(bt->graph, nullptr, &nodes);
    bt->graph_nodes = nodes;
    std::vector<cudaGraphNode_t> all(nodes);
    bt->kernel_nodes = 0;
    if (nodes && cudaGraphGetNodes(bt->graph, all.data(), &nodes) == cudaSuccess) {
        for (size_t i = 0; i < nodes; ++i) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(all[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
                bt->kernel_nodes++;
        }
    }
    bt->dirty = false;
    return BW_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace

extern "C" int bw_batch_create(bw_batch** out, void* stream, unsigned flags) {
    bw_clear_error();
    if (!out) return bw_fail(BW_EINVAL, "out is NULL");
    *out = nullptr;
    bw_batch* bt = new bw_batch();
    bt->K = (flags & BW_BATCH_THREE_PRIMES) ? 3 : 2;
    bt->persistent = (flags & BW_BATCH_PERSISTENT) != 0;
    auto fail = [&](int rc) {
        bw_batch_destroy(bt);
        return rc;
    };
    cudaError_t e = cudaSuccess;
    if (stream) {
        bt->stream = (cudaStream_t)stream;
    } else {
        e = cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking);
        bt->own_stream = true;
    }
    for (int s = 0; s < bw_batch::kSide && e == cudaSuccess; ++s) {
        e = cudaStreamCreateWithFlags(&bt->side[s], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&bt->join[s], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&bt->fork, cudaEventDisableTiming);
    for (auto& ev : bt->ev)
        if (e == cudaSuccess) e = cudaEventCreate(&ev);
    for (auto& ev : bt->chunk_ev)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&bt->d_err, 16);
    if (e == cudaSuccess) e = cudaMallocHost(&bt->h_err, 16);
    if (e != cudaSuccess) return fail(bw_fail(BW_ECUDA, "batch setup: %s", cudaGetErrorString(e)));
    *out = bt;
    return BW_OK;
}

extern "C" int bw_batch_destroy(bw_batch* bt) {
    if (!bt) return BW_OK;
    if (bt->stream) cudaStreamSynchronize(bt->stream);
    drop_layout(bt);
    cudaFree(bt->d_in);
    cudaFree(bt->d_out);
    cudaFreeHost(bt->h_in);
    cudaFreeHost(bt->h_out);
    cudaFree(bt->d_err);
    cudaFree(bt->d_qhead);
    cudaFreeHost(bt->h_err);
    for (int s = 0; s < bw_batch::kSide; ++s) {
        if (bt->side[s]) cudaStreamDestroy(bt->side[s]);
        if (bt->join[s]) cudaEventDestroy(bt->join[s]);
    }
    if (bt->fork) cudaEventDestroy(bt->fork);
    for (auto& ev : bt->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto& ev : bt->chunk_ev)
        if (ev) cudaEventDestroy(ev);
    if (bt->own_stream && bt->stream) cudaStreamDestroy(bt->stream);
    delete bt;
    return BW_OK;
}

extern "C" int bw_batch_clear(bw_batch* bt) {
    bw_clear_error();
    if (!bt) return bw_fail(BW_EINVAL, "NULL batch");
    bt->prods.clear();
    bt->dirty = true;
    return BW_OK;
}

extern "C" int bw_batch_add(bw_batch* bt, int path, const uint32_t* a, size_t la,
                            const uint32_t* b, size_t lb, uint32_t* c, size_t lc) {
    bw_clear_error();
    if (!bt || !a || !b || !c) return bw_fail(BW_EINVAL, "NULL argument");
    if (lc < la + lb) return bw_fail(BW_EINVAL, "output has %zu words, needs %zu", lc, la + lb);
    if (path == BW_PATH_AUTO) path = bw_choose_path(bt->K, la, lb);
    int log_n = 0;
    int rc = bw_check_size(path, bt->K, la, lb, &log_n);
    if (rc) return rc;
    if (log_n > kMaxGroupLogN)
        return bw_fail(BW_ESIZE, "batched products are limited to n <= 2^%d (got 2^%d)",
                       kMaxGroupLogN, log_n);
    if ((la + lb) > 0xffffffffu) return bw_fail(BW_ESIZE, "operand too long for a batch");
    Prod p;
    p.path = path;
    p.a = a;
    p.b = b;
    p.c = c;
    p.la = la;
    p.lb = lb;
    p.lc = lc;
    p.square = (a == b && la == lb);
    p.log_n = log_n;
    bt->prods.push_back(p);
    bt->dirty = true;
    return BW_OK;
}

extern "C" int bw_batch_run(bw_batch* bt, unsigned what, bw_timing* tm) {
    bw_clear_error();
    if (!bt) return bw_fail(BW_EINVAL, "NULL batch");
    if (bt->prods.empty()) return BW_OK;
    if (what == 0) what = BW_BATCH_UPLOAD | BW_BATCH_COMPUTE | BW_BATCH_DOWNLOAD;
    if (bt->dirty) {
        const int rc = build_layout(bt);
        if (rc) return rc;
        what |= BW_BATCH_UPLOAD;  // the staging arenas were (re)built
    }
    const size_t np = bt->prods.size();
    auto chunk = [&](size_t c) { return c * np / kStageChunks; };
    cudaEventRecord(bt->ev[0], bt->stream);
    if (what & BW_BATCH_UPLOAD) {
        // chunk c's DMA runs while the host stages chunk c + 1
        for (size_t c = 0; c < kStageChunks; ++c) {
            const size_t lo = chunk(c), hi = chunk(c + 1);
            if (lo == hi) continue;
            const size_t w_lo = bt->prods[lo].in_a;
            const size_t w_hi = hi < np ? bt->prods[hi].in_a : bt->in_words;
            parallel_products(lo, hi, (w_hi - w_lo) * 4, [&](size_t i) {
                const Prod& p = bt->prods[i];
                memcpy(bt->h_in + p.in_a, p.a, p.la * 4);
                if (!p.square) memcpy(bt->h_in + p.in_b, p.b, p.lb * 4);
            });
            BW_TRY(cudaMemcpyAsync(bt->d_in + w_lo, bt->h_in + w_lo, (w_hi - w_lo) * 4,
                                   cudaMemcpyHostToDevice, bt->stream));
        }
    }
    cudaEventRecord(bt->ev[1], bt->stream);
    if (what & BW_BATCH_COMPUTE) BW_TRY(cudaGraphLaunch(bt->exec, bt->stream));
    cudaEventRecord(bt->ev[2], bt->stream);
    if (what & BW_BATCH_DOWNLOAD) {
        for (size_t c = 0; c < kStageChunks; ++c) {
            const size_t lo = chunk(c), hi = chunk(c + 1);
            if (lo == hi) continue;
            const size_t w_lo = bt->prods[lo].out;
            const size_t w_hi = hi < np ? bt->prods[hi].out : bt->out_words;
            BW_TRY(cudaMemcpyAsync(bt->h_out + w_lo, bt->d_out + w_lo, (w_hi - w_lo) * 4,
                                   cudaMemcpyDeviceToHost, bt->stream));
            BW_TRY(cudaEventRecord(bt->chunk_ev[c], bt->stream));
        }
    }
    BW_TRY(cudaMemcpyAsync(bt->h_err, bt->d_err, 4, cudaMemcpyDeviceToHost, bt->stream));
    cudaEventRecord(bt->ev[3], bt->stream);
    if (what & BW_BATCH_DOWNLOAD) {
        // the host copies chunk c out while chunk c + 1 is still in flight
        for (size_t c = 0; c < kStageChunks; ++c) {
            const size_t lo = chunk(c), hi = chunk(c + 1);
            if (lo == hi) continue;
            BW_TRY(cudaEventSynchronize(bt->chunk_ev[c]));
            const size_t w_hi = hi < np ? bt->prods[hi].out : bt->out_words;
            parallel_products(lo, hi, (w_hi - bt->prods[lo].out) * 4, [&](size_t i) {
                const Prod& p = bt->prods[i];
                memcpy(p.c, bt->h_out + p.out, (p.la + p.lb) * 4);
            });
        }
    }
    BW_TRY(cudaStreamSynchronize(bt->stream));
    if (tm) {
        memset(tm, 0, sizeof *tm);
        tm->h2d_ms = elapsed(bt->ev[0], bt->ev[1]);
        tm->mul_ms = elapsed(bt->ev[1], bt->ev[2]);
        tm->d2h_ms = elapsed(bt->ev[2], bt->ev[3]);
        tm->total_ms = elapsed(bt->ev[0], bt->ev[3]);
    }
    const uint32_t err = *bt->h_err;
    if (err & 1u) return bw_fail(BW_ETIMEOUT, "carry look-back wait exceeded its bound");
    if (err) return bw_fail(BW_ECHECK, "redundant-prime reconstruction check failed");
    return BW_OK;
}

extern "C" int bw_batch_set_wait_limit(bw_batch* bt, int polls) {
    bw_clear_error();
    if (!bt || polls < 0) return bw_fail(BW_EINVAL, "bad argument");
    bt->spin_limit = polls;
    bt->dirty = true;  // the limit is a launch argument of the captured graph
    return BW_OK;
}

extern "C" int bw_batch_inject_wait_fault(bw_batch* bt, int enable) {
    bw_clear_error();
    if (!bt) return bw_fail(BW_EINVAL, "NULL batch");
    bt->inject_wait_fault = enable != 0;
    bt->dirty = true;
    return BW_OK;
}

extern "C" int bw_batch_get_info(const bw_batch* bt, bw_batch_info* o) {
    if (!bt || !o) return bw_fail(BW_EINVAL, "NULL argument");
    memset(o, 0, sizeof *o);
    o->products = bt->prods.size();
    o->buckets = bt->buckets.size();
    o->graph_nodes = bt->graph_nodes;
    o->kernel_nodes = bt->kernel_nodes;
    size_t bytes = (bt->in_cap + bt->out_cap) * 4;
    for (const Bucket& b : bt->buckets) {
        const size_t n = (size_t)1 << b.log_n;
        const int w = b.path == BW_PATH_P64 ? 8 : 4;
        bytes += b.prods.size() * b.K * n * w * (b.small ? 1 : 2) + b.plan.table_bytes;
        if (b.small) o->small_buckets++;
    }
    o->device_bytes = bytes;
    return BW_OK;
}

// Time every candidate form of every bucket on the batch's own products and
// keep the fastest in the tune table.
extern "C" int bw_batch_autotune(bw_batch* bt, int reps) {
    bw_clear_error();
    if (!bt) return bw_fail(BW_EINVAL, "NULL batch");
    if (bt->prods.empty()) return BW_OK;
    if (reps < 1) reps = 3;
    // candidate list per key
    std::map<TuneKey, std::vector<TuneVal>> cands;
    for (const Prod& p : bt->prods) {
        TuneKey key{p.path, bt->K, p.log_n};
        if (cands.count(key)) continue;
        std::vector<TuneVal> v;
        if (p.log_n <= small_max_log(p.path)) v.push_back(TuneVal{1, 0, 0, 0.f});
        // 4-step splits from square to long rows (columns of 2^2 at least),
        // each with row rounds of radix 8 and of radix 16
        const int max_c = p.path == BW_PATH_P64 ? 13 : 14;
        for (int lc = (p.log_n + 1) / 2 - 1; lc <= std::min(max_c, p.log_n - 2); ++lc)
            if (lc >= 2 && p.log_n - lc <= 13)
                for (int rl = 3; rl <= 4; ++rl) v.push_back(TuneVal{0, lc, rl, 0.f});
        cands[key] = v;
    }
    // one sub-batch per key with the batch's products of that key
    for (auto& kv : cands) {
        const TuneKey key = kv.first;
        TuneVal best{0, 0, 0, 1e30f};
        for (const TuneVal& cand : kv.second) {
            {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                g_tune[key] = cand;
            }
            bw_batch* sub = nullptr;
            int rc = bw_batch_create(&sub, nullptr, bt->K == 3 ? BW_BATCH_THREE_PRIMES : 0);
            if (rc) return rc;
            for (const Prod& p : bt->prods)
                if (p.path == key.path && p.log_n == key.log_n)
                    bw_batch_add(sub, p.path, p.a, p.la, p.b, p.lb, p.c, p.lc);
            rc = bw_batch_run(sub, BW_BATCH_UPLOAD | BW_BATCH_COMPUTE, nullptr);
            float ms = 1e30f;
            for (int r = 0; r < reps && !rc; ++r) {
                bw_timing t;
                rc = bw_batch_run(sub, BW_BATCH_COMPUTE, &t);
                ms = std::min(ms, t.mul_ms);
            }
            bw_batch_destroy(sub);
            if (rc) return rc;
            if (ms < best.ms) {
                best = cand;
                best.ms = ms;
            }
        }
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = best;
    }
    bt->dirty = true;
    return BW_OK;
}

extern "C" int bw_tune_table_export(char* buf, size_t len, size_t* needed) {
    std::string s = "[";
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        bool first = true;
        for (const auto& kv : g_tune) {
            char line[200];
            snprintf(line, sizeof line,
                     "%s{\"path\": %d, \"num_primes\": %d, \"log_n\": %d, \"small\": %d, "
                     "\"log_cols\": %d, \"row_radix\": %d, \"ms\": %.6f}",
                     first ? "" : ", ", kv.first.path, kv.first.K, kv.first.log_n,
                     kv.second.small, kv.second.log_cols,
                     kv.second.rlog ? 1 << kv.second.rlog : 0, kv.second.ms);
            s += line;
            first = false;
        }
    }
    s += "]";
    if (needed) *needed = s.size() + 1;
    if (buf && len) {
        const size_t m = std::min(len - 1, s.size());
        memcpy(buf, s.data(), m);
        buf[m] = '\0';
    }
    return BW_OK;
}

extern "C" int bw_tune_table_set(int path, int num_primes, int log_n, int small, int log_cols,
                                 int row_radix) {
    bw_clear_error();
    if (path != BW_PATH_P32 && path != BW_PATH_P64) return bw_fail(BW_EINVAL, "bad path");
    if (row_radix != 0 && row_radix != 8 && row_radix != 16)
        return bw_fail(BW_EINVAL, "row_radix must be 0 (the path's default), 8 or 16");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[TuneKey{path, num_primes == 0 ? 2 : num_primes, log_n}] =
        TuneVal{small ? 1 : 0, log_cols, row_radix == 8 ? 3 : row_radix == 16 ? 4 : 0, 0.f};
    return BW_OK;
}
