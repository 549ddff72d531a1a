// bw_server.cu -- serving engine for multiply requests (bw_server_* in
// birdwing.h).
//
// Requests arrive from any host thread (bw_server_submit) with host operand
// and result buffers.  Two native threads run the engine:
//
//   engine     admits pending requests in arrival order while the device
//              bytes they need fit the budget (admission by HBM bytes),
//              groups the admitted requests by (path, K, transform length)
//              and issues each group as one batched launch on one of several
//              CUDA streams ("lanes"): pinned staging -> one H2D copy ->
//              batched kernels -> one D2H copy.  At most max_groups_in_flight
//              groups are on the device; while that many are running, newly
//              arrived requests wait and are admitted together into the next
//              groups as earlier ones finish (continuous batching), so under
//              load the launches grow and their work overlaps on the device.
//   completer  polls the groups' completion events (any order), copies each
//              result from pinned staging into the caller's buffer, returns
//              the group's device and pinned memory and wakes waiters.
//
// Twiddle tables stay resident: one plan per (path, K, transform length,
// kernel form), built on first use or by bw_server_prewarm.  Operands,
// residues and look-back state live in one stream-ordered device block per
// group (cudaMallocAsync / cudaFreeAsync from the device's memory pool, kept
// reserved between groups).  Per-request timestamps (submit, admit, launch,
// done) give the latency distribution.
//
// The reference serves nothing: every product is one blocking
// host_multiply_merge call (src/host_multiply.cpp:27-86) that rebuilds its
// tables and buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/birdwing.h"
#include "bw_host.h"
#include "bw_internal.h"
#include "bw_kernels.cuh"

using namespace bw;

namespace {

using Clock = std::chrono::steady_clock;

constexpr size_t kAlign = 256;
// Operands and results at least this large move by DMA straight between the
// caller's pinned buffers and the device; smaller ones are staged, where one
// memcpy beats one more copy call.
constexpr size_t kDirectBytes = 64 * 1024;

bool is_pinned_host(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();  // pageable memory may report an error: not pinned
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}
size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Req {
    uint64_t id = 0;
    int path = 0, log_n = 0;
    const uint32_t* a = nullptr;
    const uint32_t* b = nullptr;
    uint32_t* c = nullptr;
    size_t la = 0, lb = 0;
    bool square = false;
    size_t dev_bytes = 0;   // device bytes charged at admission
    size_t pin_bytes = 0;   // pinned staging bytes
    Clock::time_point t_submit, t_admit, t_launch, t_done;
    int status = 1;         // 1 = not finished
    size_t group_size = 0;
    // the caller's buffers are pinned host memory (direct DMA when large)
    bool a_pin = false, b_pin = false, c_pin = false, c_direct = false;
    // offsets inside the group's device block (words); off_c_pin: the
    // result's offset in the pinned staging block when it is staged
    size_t off_a = 0, off_b = 0, off_c = 0, off_c_pin = 0;
};

// Pinned host blocks by power-of-two size class, cached for reuse; the
// total held is bounded by the staging budget.
class PinnedPool {
  public:
    explicit PinnedPool(size_t cap) : cap_(cap) {}
    ~PinnedPool() { release_all(); }
    static size_t cls(size_t bytes) {
        size_t c = 4096;
        while (c < bytes) c <<= 1;
        return c;
    }
    // nullptr when the budget is exhausted
    void* get(size_t bytes, size_t* got) {
        const size_t c = cls(bytes);
        auto& fl = free_[c];
        if (!fl.empty()) {
            void* p = fl.back();
            fl.pop_back();
            *got = c;
            return p;
        }
        // make room by dropping cached blocks of other classes
        for (auto it = free_.begin(); held_ + c > cap_ && it != free_.end(); ++it) {
            while (!it->second.empty() && held_ + c > cap_) {
                cudaFreeHost(it->second.back());
                it->second.pop_back();
                held_ -= it->first;
            }
        }
        if (held_ + c > cap_) return nullptr;
        void* p = nullptr;
        if (cudaMallocHost(&p, c) != cudaSuccess) return nullptr;
        held_ += c;
        *got = c;
        return p;
    }
    void put(void* p, size_t c) { free_[c].push_back(p); }
    void release_all() {
        for (auto& kv : free_)
            for (void* p : kv.second) cudaFreeHost(p);
        free_.clear();
        held_ = 0;
    }
    size_t cap() const { return cap_; }

  private:
    size_t cap_, held_ = 0;
    std::map<size_t, std::vector<void*>> free_;
};

struct PlanKey {
    int path, K, log_n, small, log_cols;
    bool operator<(const PlanKey& o) const {
        return std::tie(path, K, log_n, small, log_cols) <
               std::tie(o.path, o.K, o.log_n, o.small, o.log_cols);
    }
};

struct Group {
    std::vector<Req*> reqs;
    const bw_plan* plan = nullptr;
    int lane = 0;
    unsigned char* dmem = nullptr;
    unsigned char* pin = nullptr;
    size_t pin_cls = 0;
    size_t dev_bytes = 0;
    size_t err_off = 0, err_pin = 0, out_bytes = 0;
    cudaEvent_t ev = nullptr;
    int launch_status = BW_OK;
};

double us_since(Clock::time_point t0, Clock::time_point t) {
    return std::chrono::duration<double, std::micro>(t - t0).count();
}

}  // namespace

struct bw_server {
    int device = 0;
    int K = 2;
    int default_path = BW_PATH_P64;
    size_t budget = 0;
    int max_groups = 0;
    std::vector<cudaStream_t> lanes;
    int next_lane = 0;
    PinnedPool* pinned = nullptr;
    Clock::time_point t0;

    std::mutex mu;
    std::condition_variable cv_engine;    // pending work or capacity freed
    std::condition_variable cv_complete;  // groups in flight
    std::condition_variable cv_done;      // requests finished
    bool stop = false;
    std::deque<Req*> pending;
    std::unordered_map<uint64_t, Req*> reqs;  // every unreleased request
    std::deque<Req*> finished;                // not yet harvested or waited for
    std::vector<Group*> in_flight;
    std::vector<cudaEvent_t> free_events;
    uint64_t next_id = 1;
    size_t bytes_in_flight = 0, peak_bytes = 0, pinned_in_flight = 0;
    size_t launching = 0;  // requests admitted whose group is not yet in flight
    uint64_t submitted = 0, completed = 0, rejected = 0, failed = 0, groups = 0, launches = 0;
    size_t max_group = 0;

    std::mutex plan_mu;
    std::map<PlanKey, bw_plan*> plans;
    std::atomic<size_t> plan_bytes{0};

    std::thread engine, completer;
};

namespace {

bool small_form(int path, int K, int log_n, int* log_cols) {
    int small = 0;
    bw_tune_lookup(path, K, log_n, &small, log_cols);
    return small != 0;
}

size_t res_elems_bytes(int path, int K, int log_n) {
    return (size_t)K * ((size_t)1 << log_n) * (path == BW_PATH_P64 ? 8 : 4);
}

// Device bytes one request needs inside a group block.
size_t request_bytes(int path, int K, int log_n, size_t la, size_t lb, bool square) {
    int lc = 0;
    const bool small = small_form(path, K, log_n, &lc);
    const size_t words = la + lb;
    const size_t ntiles = bw_group_ntiles(path, log_n, words);
    size_t b = sizeof(BatchProd) + 4 * align_up(la, 4) + (square ? 0 : 4 * align_up(lb, 4)) +
               4 * align_up(words, 4) + res_elems_bytes(path, K, log_n) * (small ? 1 : 2);
    if (!small) b += bw_group_state_stride(ntiles);
    return b + kAlign;
}

int get_plan(bw_server* s, int path, int log_n, bw_plan** out) {
    int log_cols = 0;
    const int small = small_form(path, s->K, log_n, &log_cols) ? 1 : 0;
    const PlanKey key{path, s->K, log_n, small, log_cols};
    std::lock_guard<std::mutex> lk(s->plan_mu);
    auto it = s->plans.find(key);
    if (it != s->plans.end()) {
        *out = it->second;
        return BW_OK;
    }
    bw_plan* pl = new bw_plan();
    const int rc = bw_plan_setup(pl, path, s->K, log_n, BW_PLAN_LOG_COLS(log_cols), small);
    if (rc) {
        delete pl;
        return rc;
    }
    s->plans[key] = pl;
    s->plan_bytes += pl->table_bytes;
    *out = pl;
    return BW_OK;
}

// Finish every request of a group with one status (engine or completer).
void finish_group_locked(bw_server* s, Group* g, int status, Clock::time_point t) {
    for (Req* r : g->reqs) {
        r->status = status;
        r->t_done = t;
        s->finished.push_back(r);
        if (status == BW_OK) {
            ++s->completed;
        } else {
            ++s->failed;
        }
    }
}

// Lay out, stage and issue one group on its lane.  Called without the lock.
int launch_group(bw_server* s, Group* g) {
    const Req* r0 = g->reqs[0];
    const int path = r0->path, log_n = r0->log_n;
    bw_plan* pl = nullptr;
    int rc = get_plan(s, path, log_n, &pl);
    if (rc) return rc;
    g->plan = pl;
    const bool small = pl->small != 0;
    const size_t np = g->reqs.size();
    size_t max_words = 0;
    for (const Req* r : g->reqs) max_words = std::max(max_words, r->la + r->lb);
    const size_t ntiles = bw_group_ntiles(path, log_n, max_words);
    // Device block: [desc | staged inputs | direct inputs | err | staged
    // outputs | direct outputs | states | res_a | res_b].  The pinned staging
    // block holds [desc | staged inputs] and [err | staged outputs], so one
    // H2D and one D2H copy move every staged operand and result; operands and
    // results in the caller's own pinned memory (large ones) move by DMA
    // straight from and to it.
    auto direct = [](bool pinned, size_t words) { return pinned && words * 4 >= kDirectBytes; };
    size_t off = align_up(np * sizeof(BatchProd), 16);
    for (Req* r : g->reqs) {
        if (!direct(r->a_pin, r->la)) {
            r->off_a = off / 4;
            off += 4 * align_up(r->la, 4);
        }
        if (!r->square && !direct(r->b_pin, r->lb)) {
            r->off_b = off / 4;
            off += 4 * align_up(r->lb, 4);
        }
    }
    const size_t staged_in_end = off;
    for (Req* r : g->reqs) {
        if (direct(r->a_pin, r->la)) {
            r->off_a = off / 4;
            off += 4 * align_up(r->la, 4);
        }
        if (!r->square && direct(r->b_pin, r->lb)) {
            r->off_b = off / 4;
            off += 4 * align_up(r->lb, 4);
        }
        if (r->square) r->off_b = r->off_a;
    }
    g->err_off = off;
    off += 16;
    size_t pin_off = staged_in_end;  // err + staged outputs follow the inputs
    g->err_pin = pin_off;
    pin_off += 16;
    for (Req* r : g->reqs) {
        if (!direct(r->c_pin, r->la + r->lb)) {
            r->off_c = off / 4;
            r->off_c_pin = pin_off / 4;
            off += 4 * align_up(r->la + r->lb, 4);
            pin_off += 4 * align_up(r->la + r->lb, 4);
        }
    }
    g->out_bytes = off - g->err_off - 16;  // staged outputs only
    for (Req* r : g->reqs) {
        if (direct(r->c_pin, r->la + r->lb)) {
            r->off_c = off / 4;
            r->c_direct = true;
            off += 4 * align_up(r->la + r->lb, 4);
        }
    }
    const size_t st_stride = small ? 0 : bw_group_state_stride(ntiles);
    const size_t st_off = align_up(off, 16);
    off = align_up(st_off + np * st_stride, kAlign);
    const size_t per = res_elems_bytes(path, s->K, log_n);
    const size_t ra_off = off;
    off += np * per;
    const size_t rb_off = off;
    if (!small) off += np * per;
    g->dev_bytes = off;
    const size_t pin_need = pin_off;

    {
        std::lock_guard<std::mutex> lk(s->mu);
        g->pin = static_cast<unsigned char*>(s->pinned->get(pin_need, &g->pin_cls));
    }
    if (!g->pin) return bw_fail(BW_ENOMEM, "pinned staging exhausted");
    cudaStream_t st = s->lanes[g->lane];
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&g->dmem), g->dev_bytes, st);
    if (e != cudaSuccess) return bw_fail(BW_ENOMEM, "cudaMallocAsync: %s", cudaGetErrorString(e));
    // descriptors and staged operands into pinned staging
    BatchProd* desc = reinterpret_cast<BatchProd*>(g->pin);
    uint32_t* hw = reinterpret_cast<uint32_t*>(g->pin);
    uint32_t* dw = reinterpret_cast<uint32_t*>(g->dmem);
    for (size_t q = 0; q < np; ++q) {
        Req* r = g->reqs[q];
        if (!direct(r->a_pin, r->la)) memcpy(hw + r->off_a, r->a, r->la * 4);
        if (!r->square && !direct(r->b_pin, r->lb)) memcpy(hw + r->off_b, r->b, r->lb * 4);
        BatchProd d{};
        d.a = dw + r->off_a;
        d.b = dw + r->off_b;
        d.out = dw + r->off_c;
        d.la = (uint32_t)r->la;
        d.lb = (uint32_t)r->lb;
        d.square = r->square ? 1u : 0u;
        d.res_off = q * (per / (path == BW_PATH_P64 ? 8 : 4));
        if (!small) bw_group_fill_state(d, g->dmem + st_off + q * st_stride, ntiles);
        desc[q] = d;
    }
    const auto t_launch = Clock::now();
    for (Req* r : g->reqs) r->t_launch = t_launch;
    e = cudaMemcpyAsync(g->dmem, g->pin, staged_in_end, cudaMemcpyHostToDevice, st);
    for (Req* r : g->reqs) {
        if (e == cudaSuccess && direct(r->a_pin, r->la))
            e = cudaMemcpyAsync(dw + r->off_a, r->a, r->la * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && !r->square && direct(r->b_pin, r->lb))
            e = cudaMemcpyAsync(dw + r->off_b, r->b, r->lb * 4, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(g->dmem + g->err_off, 0, 16, st);
    if (e == cudaSuccess && !small)
        e = cudaMemsetAsync(g->dmem + st_off, 0, np * st_stride, st);
    if (e != cudaSuccess) return bw_fail(BW_ECUDA, "staging: %s", cudaGetErrorString(e));
    bw_group_launch gl{pl,
                       reinterpret_cast<const BatchProd*>(g->dmem),
                       (unsigned)np,
                       g->dmem + ra_off,
                       small ? nullptr : g->dmem + rb_off,
                       ntiles,
                       reinterpret_cast<uint32_t*>(g->dmem + g->err_off),
                       1 << 22,
                       false};
    rc = bw_enqueue_group(gl, st);
    if (rc) return rc;
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->pin + g->err_pin, g->dmem + g->err_off, 16 + g->out_bytes,
                            cudaMemcpyDeviceToHost, st);
    for (Req* r : g->reqs)
        if (e == cudaSuccess && r->c_direct)
            e = cudaMemcpyAsync(r->c, dw + r->off_c, (r->la + r->lb) * 4, cudaMemcpyDeviceToHost,
                                st);
    if (e == cudaSuccess) {
        e = cudaFreeAsync(g->dmem, st);
        if (e == cudaSuccess) g->dmem = nullptr;  // released in stream order
    }
    if (e == cudaSuccess) e = cudaEventRecord(g->ev, st);
    if (e != cudaSuccess) return bw_fail(BW_ECUDA, "launch: %s", cudaGetErrorString(e));
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->launches += small ? 1 : 4;
    }
    return BW_OK;
}

void engine_loop(bw_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_engine.wait(lk, [&] {
            return s->stop ||
                   (!s->pending.empty() && (int)s->in_flight.size() < s->max_groups);
        });
        if (s->stop) break;
        // admit in arrival order while the bytes fit
        std::vector<Req*> take;
        size_t bytes = 0, pin = 0;
        const size_t plan_b = s->plan_bytes.load();
        while (!s->pending.empty()) {
            Req* r = s->pending.front();
            if (s->bytes_in_flight + plan_b + bytes + r->dev_bytes > s->budget) break;
            if (s->pinned_in_flight + pin + r->pin_bytes > s->pinned->cap()) break;
            bytes += r->dev_bytes;
            pin += r->pin_bytes;
            take.push_back(r);
            s->pending.pop_front();
        }
        if (take.empty()) {
            // the head does not fit yet: wait for a completion
            if (s->in_flight.empty()) {
                // nothing will free memory: the request can never run
                Req* r = s->pending.front();
                s->pending.pop_front();
                r->status = BW_EREJECT;
                r->t_done = Clock::now();
                ++s->rejected;
                s->finished.push_back(r);
                s->cv_done.notify_all();
            } else {
                s->cv_engine.wait(lk);
            }
            continue;
        }
        const auto t_admit = Clock::now();
        s->launching += take.size();
        s->bytes_in_flight += bytes;
        s->pinned_in_flight += pin;
        s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_flight + plan_b);
        // groups of equal (path, log_n), arrival order of their first member
        std::vector<Group*> gs;
        std::map<std::pair<int, int>, Group*> by_key;
        for (Req* r : take) {
            r->t_admit = t_admit;
            const auto key = std::make_pair(r->path, r->log_n);
            auto it = by_key.find(key);
            if (it == by_key.end() || it->second->reqs.size() >= 16384) {
                Group* g = new Group();
                gs.push_back(g);
                by_key[key] = g;
                it = by_key.find(key);
            }
            it->second->reqs.push_back(r);
        }
        for (Group* g : gs) {
            g->lane = s->next_lane;
            s->next_lane = (s->next_lane + 1) % (int)s->lanes.size();
            if (!s->free_events.empty()) {
                g->ev = s->free_events.back();
                s->free_events.pop_back();
            } else {
                cudaEventCreateWithFlags(&g->ev, cudaEventDisableTiming);
            }
            for (Req* r : g->reqs) r->group_size = g->reqs.size();
        }
        lk.unlock();
        for (Group* g : gs) g->launch_status = launch_group(s, g);
        lk.lock();
        for (Group* g : gs) {
            ++s->groups;
            s->max_group = std::max(s->max_group, g->reqs.size());
            s->in_flight.push_back(g);
        }
        s->launching -= take.size();
        s->cv_complete.notify_all();
    }
}

void complete_group(bw_server* s, Group* g) {
    int status = g->launch_status;
    if (status == BW_OK) {
        const cudaError_t e = cudaEventSynchronize(g->ev);
        if (e != cudaSuccess) {
            status = BW_ECUDA;
        } else {
            uint32_t err = 0;
            memcpy(&err, g->pin + g->err_pin, 4);
            if (err & 1u) {
                status = BW_ETIMEOUT;
            } else if (err) {
                status = BW_ECHECK;
            }
        }
        if (status == BW_OK) {
            const uint32_t* hw = reinterpret_cast<const uint32_t*>(g->pin);
            for (Req* r : g->reqs)
                if (!r->c_direct) memcpy(r->c, hw + r->off_c_pin, (r->la + r->lb) * 4);
        }
    } else {
        // the launch failed part way: let what was enqueued finish
        cudaStreamSynchronize(s->lanes[g->lane]);
        if (g->dmem) cudaFree(g->dmem);
    }
    const auto t = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    size_t bytes = 0, pin = 0;
    for (Req* r : g->reqs) {
        bytes += r->dev_bytes;
        pin += r->pin_bytes;
    }
    s->bytes_in_flight -= bytes;
    s->pinned_in_flight -= pin;
    if (g->pin) s->pinned->put(g->pin, g->pin_cls);
    if (g->ev) s->free_events.push_back(g->ev);
    finish_group_locked(s, g, status, t);
    s->in_flight.erase(std::find(s->in_flight.begin(), s->in_flight.end(), g));
    delete g;
    s->cv_done.notify_all();
    s->cv_engine.notify_all();
}

void completer_loop(bw_server* s) {
    cudaSetDevice(s->device);
    int idle_polls = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_complete.wait(lk, [&] { return s->stop || !s->in_flight.empty(); });
        if (s->in_flight.empty() && s->stop) break;
        std::vector<Group*> snap = s->in_flight;
        lk.unlock();
        Group* ready = nullptr;
        for (Group* g : snap) {
            if (g->launch_status != BW_OK || cudaEventQuery(g->ev) != cudaErrorNotReady) {
                ready = g;
                break;
            }
        }
        if (ready) {
            complete_group(s, ready);
            idle_polls = 0;
        } else if (++idle_polls < 20000) {
            std::this_thread::yield();  // a finished group is seen within microseconds
        } else {
            std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
        lk.lock();
    }
}

void fill_info(const bw_server* s, const Req* r, bw_request_info* o) {
    memset(o, 0, sizeof *o);
    o->ticket = r->id;
    o->status = r->status;
    o->submit_us = us_since(s->t0, r->t_submit);
    o->admit_us = r->t_admit.time_since_epoch().count() ? us_since(s->t0, r->t_admit) : -1.0;
    o->launch_us = r->t_launch.time_since_epoch().count() ? us_since(s->t0, r->t_launch) : -1.0;
    o->done_us = us_since(s->t0, r->t_done);
    o->group_size = r->group_size;
    o->device_bytes = r->dev_bytes;
    o->la = r->la;
    o->lb = r->lb;
}

}  // namespace

extern "C" int bw_server_create(bw_server** out, const bw_server_config* cfg) {
    bw_clear_error();
    if (!out) return bw_fail(BW_EINVAL, "out is NULL");
    *out = nullptr;
    bw_server_config c{};
    if (cfg) c = *cfg;
    if (c.num_primes != 0 && c.num_primes != 2 && c.num_primes != 3)
        return bw_fail(BW_EINVAL, "num_primes must be 2 or 3");
    if (c.path != BW_PATH_AUTO && c.path != BW_PATH_P32 && c.path != BW_PATH_P64)
        return bw_fail(BW_EINVAL, "unknown path %d", c.path);
    bw_server* s = new bw_server();
    s->K = c.num_primes ? c.num_primes : 2;
    s->default_path = c.path;  // BW_PATH_AUTO: chosen per request
    s->budget = c.hbm_budget_bytes ? c.hbm_budget_bytes : (size_t)120 << 30;
    const int nl = c.lanes > 0 ? std::min(c.lanes, 64) : 8;
    s->max_groups = c.max_groups_in_flight > 0 ? c.max_groups_in_flight : 2 * nl;
    s->pinned = new PinnedPool(c.pinned_bytes ? c.pinned_bytes : (size_t)2 << 30);
    s->t0 = Clock::now();
    cudaError_t e = cudaGetDevice(&s->device);
    for (int i = 0; i < nl && e == cudaSuccess; ++i) {
        cudaStream_t st = nullptr;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) s->lanes.push_back(st);
    }
    if (e == cudaSuccess) {
        // keep freed group blocks reserved in the device pool between groups
        cudaMemPool_t pool;
        e = cudaDeviceGetDefaultMemPool(&pool, s->device);
        if (e == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    if (e != cudaSuccess) {
        const int rc = bw_fail(BW_ECUDA, "server setup: %s", cudaGetErrorString(e));
        bw_server_destroy(s);
        return rc;
    }
    s->engine = std::thread(engine_loop, s);
    s->completer = std::thread(completer_loop, s);
    *out = s;
    return BW_OK;
}

extern "C" int bw_server_destroy(bw_server* s) {
    if (!s) return BW_OK;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        // requests not yet admitted fail; admitted ones finish
        while (!s->pending.empty()) {
            Req* r = s->pending.front();
            s->pending.pop_front();
            r->status = BW_EBUSY;
            r->t_done = Clock::now();
            ++s->failed;
            s->finished.push_back(r);
        }
        s->cv_done.notify_all();
        s->stop = true;
    }
    // the engine stops launching; the completer finishes what is in flight
    s->cv_engine.notify_all();
    if (s->engine.joinable()) s->engine.join();
    s->cv_complete.notify_all();
    if (s->completer.joinable()) s->completer.join();
    for (;;) {
        Group* g = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->in_flight.empty()) break;
            g = s->in_flight.front();
        }
        complete_group(s, g);
    }
    for (cudaStream_t st : s->lanes) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (cudaEvent_t ev : s->free_events) cudaEventDestroy(ev);
    for (auto& kv : s->plans) {
        cudaFree(kv.second->d_tables);
        delete kv.second;
    }
    for (auto& kv : s->reqs) delete kv.second;
    delete s->pinned;
    delete s;
    return BW_OK;
}

extern "C" int bw_server_prewarm(bw_server* s, int path, int max_log_n) {
    bw_clear_error();
    if (!s) return bw_fail(BW_EINVAL, "NULL server");
    if (path == BW_PATH_AUTO) path = s->default_path;
    if (path != BW_PATH_AUTO && path != BW_PATH_P32 && path != BW_PATH_P64)
        return bw_fail(BW_EINVAL, "bad path");
    // AUTO: both paths' lengths up to max_log_n
    for (const int pth : {BW_PATH_P32, BW_PATH_P64}) {
        if (path != BW_PATH_AUTO && path != pth) continue;
        int top = std::min(max_log_n, std::min(kMaxGroupLogN, bw_path_max_log_n(pth, s->K)));
        for (int ln = 4; ln <= top; ++ln) {
            bw_plan* pl = nullptr;
            const int rc = get_plan(s, pth, ln, &pl);
            if (rc) return rc;
        }
    }
    return BW_OK;
}

extern "C" int bw_server_submit(bw_server* s, int path, const uint32_t* a, size_t la,
                                const uint32_t* b, size_t lb, uint32_t* c, size_t lc,
                                uint64_t* ticket) {
    bw_clear_error();
    if (!s || !a || !b || !c || !ticket) return bw_fail(BW_EINVAL, "NULL argument");
    if (lc < la + lb) return bw_fail(BW_EINVAL, "output has %zu words, needs %zu", lc, la + lb);
    if (path == BW_PATH_AUTO) path = s->default_path;
    if (path == BW_PATH_AUTO) path = bw_choose_path(s->K, la, lb);
    int log_n = 0;
    int rc = bw_check_size(path, s->K, la, lb, &log_n);
    if (rc) return rc;
    if (log_n > kMaxGroupLogN)
        return bw_fail(BW_ESIZE, "served products are limited to n <= 2^%d", kMaxGroupLogN);
    Req* r = new Req();
    r->path = path;
    r->log_n = log_n;
    r->a = a;
    r->b = b;
    r->c = c;
    r->la = la;
    r->lb = lb;
    r->square = (a == b && la == lb);
    r->a_pin = is_pinned_host(a);
    r->b_pin = r->square ? r->a_pin : is_pinned_host(b);
    r->c_pin = is_pinned_host(c);
    r->dev_bytes = request_bytes(path, s->K, log_n, la, lb, r->square);
    // staging charge: a group's pinned block is its bytes rounded up to a
    // power of two (at least 4 KiB), so twice the request's own bytes covers
    // its share of any group it joins
    const size_t raw = sizeof(BatchProd) + 4 * (align_up(la, 4) + align_up(lb, 4) +
                                                align_up(la + lb, 4)) + 64;
    r->pin_bytes = std::max<size_t>(4096, 2 * raw);
    if (r->dev_bytes + s->plan_bytes.load() > s->budget || r->pin_bytes > s->pinned->cap()) {
        delete r;
        std::lock_guard<std::mutex> lk(s->mu);
        ++s->rejected;
        return bw_fail(BW_EREJECT, "request needs more device or staging memory than the "
                                   "server's budget");
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->pending.push_back(r);
        ++s->submitted;
        *ticket = r->id;
    }
    s->cv_engine.notify_one();
    return BW_OK;
}

extern "C" int bw_server_wait(bw_server* s, uint64_t ticket, int timeout_ms,
                              bw_request_info* info) {
    bw_clear_error();
    if (!s) return bw_fail(BW_EINVAL, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return bw_fail(BW_EINVAL, "unknown ticket %llu",
                                            (unsigned long long)ticket);
    Req* r = it->second;
    auto done = [&] { return r->status != 1; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, done);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
        return bw_fail(BW_ETIMEOUT, "request %llu not finished", (unsigned long long)ticket);
    }
    if (info) fill_info(s, r, info);
    const int st = r->status;
    s->reqs.erase(it);
    s->finished.erase(std::find(s->finished.begin(), s->finished.end(), r));
    delete r;
    if (st != BW_OK)
        return bw_fail(st, "request %llu failed (%d)", (unsigned long long)ticket, st);
    return BW_OK;
}

extern "C" int bw_server_harvest(bw_server* s, bw_request_info* out, size_t max, size_t* count) {
    bw_clear_error();
    if (!s || !count || (max && !out)) return bw_fail(BW_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    size_t n = 0;
    while (n < max && !s->finished.empty()) {
        Req* r = s->finished.front();
        s->finished.pop_front();
        fill_info(s, r, &out[n++]);
        s->reqs.erase(r->id);
        delete r;
    }
    *count = n;
    return BW_OK;
}

extern "C" int bw_server_drain(bw_server* s, int timeout_ms) {
    bw_clear_error();
    if (!s) return bw_fail(BW_EINVAL, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [&] { return s->pending.empty() && s->launching == 0 && s->in_flight.empty(); };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, idle);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle)) {
        return bw_fail(BW_ETIMEOUT, "server not idle");
    }
    return BW_OK;
}

extern "C" int bw_server_get_stats(bw_server* s, bw_server_stats* o) {
    if (!s || !o) return bw_fail(BW_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(o, 0, sizeof *o);
    o->submitted = s->submitted;
    o->completed = s->completed;
    o->rejected = s->rejected;
    o->failed = s->failed;
    o->groups = s->groups;
    o->kernel_launches = s->launches;
    o->max_group_size = s->max_group;
    o->bytes_in_flight = s->bytes_in_flight;
    o->peak_bytes_in_flight = s->peak_bytes;
    o->resident_plan_bytes = s->plan_bytes.load();
    o->queue_depth = s->pending.size();
    o->groups_in_flight = s->in_flight.size();
    o->budget_bytes = s->budget;
    return BW_OK;
}
