// server.cu - build server: continuous batching of build requests under an HBM budget.
//
// The reference builds one scene per awaited call (scripts/bvh/build-bvh.js:12-66 from
// scripts/main.js:88).  A server keeps many such builds going: clients submit requests from
// any thread; one scheduler thread forms batches and runs them through lvbh_build_batched on
// `slots` contexts, each with its own stream, so that the copies and kernels of one batch
// overlap those of the batches already on the GPU.
//
//   * Memory.  One cudaMalloc of the budget, minus what the slot contexts hold, is carved by a
//     host-side first-fit allocator into per-batch result blocks (nodes, sorted triangles,
//     parents, leaf indices, keys of every request of the batch).  A block is returned when the
//     last of its requests is released.  Nothing is allocated on the request path, so no
//     request waits on cudaMalloc / cudaFree (both synchronise the device).
//   * Admission.  When a slot is free the scheduler takes queued requests in arrival order
//     while the batch stays within max_batch_tris / max_batch_reqs and its result block fits
//     the free memory; a batch that does not fit waits until a release frees memory.
//   * Launch.  A batch of one request is built by lvbh_build_soup straight from the request's
//     triangles (device input) or from the slot's staging buffer (host input); a batch of
//     several is staged contiguously and built by lvbh_build_batched.  Both give identical
//     trees.
//   * Completion.  An event is recorded after each batch.  While batches are in flight the
//     scheduler polls their events (yielding between polls); with nothing in flight it sleeps
//     on a condition variable until a submit or a release.  It then reads the build status and
//     publishes the results; a request's latency ends at that publication.  A batch whose
//     build reports bad input (a non-finite vertex) is rebuilt request by request so that only
//     the offending requests fail.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "lvbh.h"
#include "lvbh_internal.h"

namespace {

using Clock = std::chrono::steady_clock;
constexpr size_t kGranule = 256;
inline size_t round_up(size_t x) { return (x + kGranule - 1) & ~(kGranule - 1); }
inline double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// First-fit allocator of byte ranges of one device reservation; freed ranges merge with their
// neighbours.
class RangeAlloc {
  public:
    void reset(size_t cap) {
        free_.clear();
        used_ = peak_ = 0;
        if (cap) free_[0] = cap;
    }
    bool alloc(size_t bytes, size_t *off) {
        bytes = round_up(bytes ? bytes : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used_ += bytes;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = round_up(bytes ? bytes : 1);
        used_ -= bytes;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + bytes == next->first) {
            bytes += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }

  private:
    std::map<size_t, size_t> free_;
    size_t used_ = 0, peak_ = 0;
};

// Byte layout of the results of `t` triangles: nodes, tris, parents, leaf_index, morton.
struct BlockLayout {
    size_t off[5];
    size_t bytes;
    explicit BlockLayout(uint64_t t) {
        const size_t sz[5] = {64 * t, 48 * t, 8 * t, 4 * t, 4 * t};
        size_t o = 0;
        for (int i = 0; i < 5; ++i) {
            off[i] = o;
            o += round_up(sz[i]);
        }
        bytes = o;
    }
};

struct Block {
    size_t off = 0, bytes = 0;
    uint64_t tris = 0;
    int refs = 0;
};

struct Req {
    uint64_t id = 0;
    const float *tri = nullptr;
    uint32_t n = 0;
    bool host = false, has_bounds = false;
    float bounds[6] = {0, 0, 0, 0, 0, 0};
    float out_bounds[6] = {0, 0, 0, 0, 0, 0};
    Clock::time_point t_submit, t_launch, t_done;
    int status = LVBH_EBUSY;
    uint32_t batch_reqs = 0, batch_tris = 0;
    Block *block = nullptr;
    uint64_t slice = 0;  // first triangle of this request inside its block
};

struct Slot {
    lvbh_server *srv = nullptr;
    lvbh_ctx *ctx = nullptr;
    cudaStream_t stream = nullptr;
    float *input = nullptr;  // max_batch_tris staged triangles
    std::vector<Req *> reqs;
    Block *block = nullptr;
    std::vector<uint32_t> offs;
    std::vector<float> seg_bounds, bounds_out;
    lvbh_result res{};
    cudaEvent_t ev = nullptr;
    bool busy = false;
    bool single = false;  // built with lvbh_build_soup
    int launch_rc = LVBH_OK;
};

}  // namespace

struct lvbh_server {
    int device = 0;
    uint32_t max_tris = 0, max_reqs = 0, max_requests = 0;
    size_t budget = 0;
    std::string err;
    void *arena = nullptr;
    size_t arena_bytes = 0;
    RangeAlloc alloc;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv;       // wakes the scheduler
    std::condition_variable cv_done;  // wakes clients waiting on a request
    std::deque<Req *> queue;
    std::unordered_map<uint64_t, Req *> reqs;
    uint64_t next_id = 1;
    bool stop = false, mem_blocked = false;
    std::thread th;
    lvbh_server_stats st{};
};

namespace {

// Launches the batch staged in s->reqs (scheduler thread, without the lock).
void issue(lvbh_server *srv, Slot &s) {
    const size_t m = s.reqs.size();
    s.offs.assign(m + 1, 0);
    bool any_bounds = false;
    for (size_t i = 0; i < m; ++i) {
        s.offs[i + 1] = s.offs[i] + s.reqs[i]->n;
        any_bounds |= s.reqs[i]->has_bounds;
    }
    const uint64_t total = s.offs[m];
    s.seg_bounds.clear();
    if (any_bounds) {
        s.seg_bounds.assign(6 * m, NAN);
        for (size_t i = 0; i < m; ++i)
            if (s.reqs[i]->has_bounds) std::memcpy(&s.seg_bounds[6 * i], s.reqs[i]->bounds, 24);
    }
    s.bounds_out.assign(6 * m, 0.0f);
    char *base = static_cast<char *>(srv->arena) + s.block->off;
    const BlockLayout lay(total);
    s.res = lvbh_result{};
    s.res.nodes = base + lay.off[0];
    s.res.tris = base + lay.off[1];
    s.res.parents = reinterpret_cast<int32_t *>(base + lay.off[2]);
    s.res.leaf_index = reinterpret_cast<uint32_t *>(base + lay.off[3]);
    s.res.morton = reinterpret_cast<uint32_t *>(base + lay.off[4]);
    int rc = LVBH_OK;
    s.single = m == 1;
    if (s.single) {
        const Req *r = s.reqs[0];
        const float *src = r->tri;
        if (r->host) {
            if (cudaMemcpyAsync(s.input, r->tri, 48ull * r->n, cudaMemcpyHostToDevice, s.stream) != cudaSuccess) {
                cudaGetLastError();
                rc = LVBH_ECUDA;
            }
            src = s.input;
        }
        if (rc == LVBH_OK)
            rc = lvbh_build_soup(s.ctx, src, r->n, r->has_bounds ? r->bounds : nullptr,
                                 LVBH_OUT_CALLER | LVBH_ASYNC | LVBH_NO_GRAPH, &s.res, s.stream);
    } else {
        for (size_t i = 0; i < m && rc == LVBH_OK; ++i) {
            const Req *r = s.reqs[i];
            if (!r->n) continue;
            const cudaError_t e = cudaMemcpyAsync(s.input + 12ull * s.offs[i], r->tri, 48ull * r->n,
                                                  r->host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                                  s.stream);
            if (e != cudaSuccess) { cudaGetLastError(); rc = LVBH_ECUDA; }
        }
        if (rc == LVBH_OK)
            rc = lvbh_build_batched(s.ctx, s.input, s.offs.data(), (uint32_t)m,
                                    any_bounds ? s.seg_bounds.data() : nullptr, s.bounds_out.data(),
                                    LVBH_OUT_CALLER | LVBH_ASYNC | LVBH_NO_GRAPH, &s.res, s.stream);
    }
    if (rc == LVBH_OK && cudaEventRecord(s.ev, s.stream) != cudaSuccess) {
        cudaGetLastError();
        rc = LVBH_ECUDA;
    }
    s.launch_rc = rc;
}

// Retires a finished batch (scheduler thread, without the lock).
void finish(lvbh_server *srv, Slot &s) {
    int rc = s.launch_rc;
    if (rc == LVBH_OK) rc = lvbh_sync(s.ctx);
    else cudaStreamSynchronize(s.stream);
    const size_t m = s.reqs.size();
    if (s.single) std::memcpy(s.bounds_out.data(), s.res.bounds, sizeof s.res.bounds);
    std::vector<int> status(m, rc);
    if (rc == LVBH_EINVAL && m > 1) {
        // attribute bad input: rebuild each request alone into its own slice
        for (size_t i = 0; i < m; ++i) {
            const Req *r = s.reqs[i];
            uint32_t offs[2] = {0, r->n};
            lvbh_result one{};
            const uint64_t o = s.offs[i];
            one.nodes = static_cast<char *>(s.res.nodes) + 64 * o;
            one.tris = static_cast<char *>(s.res.tris) + 48 * o;
            one.parents = s.res.parents + 2 * o;
            one.leaf_index = s.res.leaf_index + o;
            one.morton = s.res.morton + o;
            status[i] = lvbh_build_batched(s.ctx, s.input + 12 * o, offs, 1,
                                           r->has_bounds ? r->bounds : nullptr, &s.bounds_out[6 * i],
                                           LVBH_OUT_CALLER | LVBH_NO_GRAPH, &one, s.stream);
        }
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    const Clock::time_point now = Clock::now();
    for (size_t i = 0; i < m; ++i) {
        Req *r = s.reqs[i];
        r->status = status[i];
        r->t_done = now;
        std::memcpy(r->out_bounds, &s.bounds_out[6 * i], sizeof r->out_bounds);
        if (status[i] == LVBH_OK) {
            ++srv->st.completed;
            srv->st.tris_built += r->n;
        } else {
            ++srv->st.failed;
        }
    }
    s.reqs.clear();
    s.block = nullptr;
    s.busy = false;
    srv->cv_done.notify_all();
}

// Takes queued requests for a batch and reserves their result block (with the lock held).
bool form_batch(lvbh_server *srv, Slot &s) {
    uint64_t tris = 0;
    size_t take = 0;
    while (take < srv->queue.size() && take < srv->max_reqs) {
        const uint64_t n = srv->queue[take]->n;
        if (take && tris + n > srv->max_tris) break;
        tris += n;
        ++take;
    }
    // shrink until the result block fits the free memory
    size_t off = 0;
    while (take) {
        if (srv->alloc.alloc(BlockLayout(tris).bytes, &off)) break;
        --take;
        tris -= srv->queue[take]->n;
    }
    if (!take) {
        ++srv->st.admission_waits;
        srv->mem_blocked = true;
        return false;
    }
    Block *b = new Block;
    b->off = off;
    b->bytes = BlockLayout(tris).bytes;
    b->tris = tris;
    b->refs = (int)take;
    const Clock::time_point now = Clock::now();
    uint64_t at = 0;
    for (size_t i = 0; i < take; ++i) {
        Req *r = srv->queue.front();
        srv->queue.pop_front();
        r->block = b;
        r->slice = at;
        r->t_launch = now;
        r->batch_reqs = (uint32_t)take;
        r->batch_tris = (uint32_t)tris;
        at += r->n;
        s.reqs.push_back(r);
    }
    s.block = b;
    s.busy = true;
    ++srv->st.batches;
    srv->st.max_batch_seen = std::max<uint32_t>(srv->st.max_batch_seen, (uint32_t)take);
    return true;
}

// True when the slot's batch has finished on the device (or never launched).
bool slot_done(Slot &s) {
    if (s.launch_rc != LVBH_OK) return true;
    const cudaError_t e = cudaEventQuery(s.ev);
    if (e == cudaErrorNotReady) return false;
    if (e != cudaSuccess) cudaGetLastError();  // the build's own status reports the failure
    return true;
}

void scheduler(lvbh_server *srv) {
    cudaSetDevice(srv->device);
    std::unique_lock<std::mutex> lk(srv->mu);
    for (;;) {
        bool worked = false, busy = false;
        lk.unlock();  // slots are the scheduler's own: poll and retire them without the lock
        for (Slot &s : srv->slots) {
            if (s.busy && slot_done(s)) {
                finish(srv, s);
                worked = true;
            }
        }
        lk.lock();
        for (Slot &s : srv->slots) {
            if (s.busy || srv->queue.empty() || srv->mem_blocked) continue;
            if (!form_batch(srv, s)) break;
            lk.unlock();
            issue(srv, s);
            lk.lock();
            worked = true;
        }
        for (const Slot &s : srv->slots) busy |= s.busy;
        if (srv->stop && srv->queue.empty() && !busy) break;
        if (srv->stop && !busy && srv->mem_blocked) {  // nothing left can free memory
            for (Req *r : srv->queue) { r->status = LVBH_ENOMEM; r->t_done = Clock::now(); ++srv->st.failed; }
            srv->queue.clear();
            srv->cv_done.notify_all();
            break;
        }
        if (worked) continue;
        if (busy) {  // batches in flight: poll their events again after yielding the core
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
            continue;
        }
        srv->cv.wait(lk, [&] {
            return srv->stop || (!srv->queue.empty() && !srv->mem_blocked);
        });
    }
}

void fill(const lvbh_server *srv, const Req *r, lvbh_result *out, lvbh_request_info *info) {
    if (info) {
        info->status = r->status;
        info->num_tris = r->n;
        info->batch_reqs = r->batch_reqs;
        info->batch_tris = r->batch_tris;
        info->queued_ms = r->status == LVBH_EBUSY ? 0.0 : ms_between(r->t_submit, r->t_launch);
        info->latency_ms = r->status == LVBH_EBUSY ? 0.0 : ms_between(r->t_submit, r->t_done);
    }
    if (out) {
        *out = lvbh_result{};
        out->num_tris = out->num_nodes = r->n;
        std::memcpy(out->bounds, r->out_bounds, sizeof out->bounds);
        if (r->block && r->n && r->status == LVBH_OK) {
            char *base = static_cast<char *>(srv->arena) + r->block->off;
            const BlockLayout lay(r->block->tris);
            const uint64_t o = r->slice;
            out->nodes = base + lay.off[0] + 64 * o;
            out->tris = base + lay.off[1] + 48 * o;
            out->parents = reinterpret_cast<int32_t *>(base + lay.off[2]) + 2 * o;
            out->leaf_index = reinterpret_cast<uint32_t *>(base + lay.off[3]) + o;
            out->morton = reinterpret_cast<uint32_t *>(base + lay.off[4]) + o;
        }
    }
}

void destroy_slots(lvbh_server *srv) {
    for (Slot &s : srv->slots) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        if (s.ctx) lvbh_destroy(s.ctx);
        if (s.input) cudaFree(s.input);
        if (s.stream) cudaStreamDestroy(s.stream);
        if (s.ev) cudaEventDestroy(s.ev);
        s.ev = nullptr;
        s.ctx = nullptr;
        s.input = nullptr;
        s.stream = nullptr;
    }
}

}  // namespace

extern "C" {

int lvbh_server_create(lvbh_server **out, const lvbh_server_config *cfg) {
    if (!out) return LVBH_EINVAL;
    *out = nullptr;
    lvbh_server_config c{};
    c.device = -1;
    if (cfg) c = *cfg;
    const uint32_t slots = c.slots ? c.slots : 3;
    const uint64_t budget = c.hbm_budget ? c.hbm_budget : 96ull << 30;
    const uint32_t max_tris = c.max_batch_tris ? c.max_batch_tris : 1u << 24;
    const uint32_t max_reqs = c.max_batch_reqs ? c.max_batch_reqs : 4096;
    if (slots > 64 || max_tris > LVBH_MAX_TRIS || max_reqs > (1u << 24)) return LVBH_EINVAL;
    int dev = c.device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return LVBH_ECUDA; }
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(dev) != cudaSuccess) { cudaGetLastError(); return LVBH_EINVAL; }
    lvbh_server *srv = new (std::nothrow) lvbh_server();
    if (!srv) return LVBH_ENOMEM;
    srv->device = dev;
    srv->max_tris = max_tris;
    srv->max_reqs = max_reqs;
    srv->max_requests = c.max_requests ? c.max_requests : 1u << 20;
    srv->budget = budget;
    srv->slots.resize(slots);
    int rc = LVBH_OK;
    size_t held = 0;
    for (Slot &s : srv->slots) {
        s.srv = srv;
        lvbh_config lc{};
        lc.device = dev;
        if ((rc = lvbh_create(&s.ctx, &lc)) != LVBH_OK) break;
        if ((rc = lvbh::ctx_reserve_batch(s.ctx, max_tris, max_reqs)) != LVBH_OK) break;
        if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc(&s.input, 48ull * max_tris) != cudaSuccess) {
            cudaGetLastError();
            rc = LVBH_ENOMEM;
            break;
        }
        held += lvbh::ctx_device_bytes(s.ctx) + 48ull * max_tris;
    }
    if (rc == LVBH_OK && held + (64u << 20) > budget) rc = LVBH_ENOMEM;  // budget below the scratch
    if (rc == LVBH_OK) {
        srv->arena_bytes = (budget - held) & ~(kGranule - 1);
        if (cudaMalloc(&srv->arena, srv->arena_bytes) != cudaSuccess) {
            cudaGetLastError();
            srv->arena = nullptr;
            rc = LVBH_ENOMEM;
        }
    }
    if (rc != LVBH_OK) {
        destroy_slots(srv);
        delete srv;
        if (prev >= 0) cudaSetDevice(prev);
        return rc;
    }
    srv->alloc.reset(srv->arena_bytes);
    srv->st.budget_bytes = budget;
    srv->st.result_bytes = srv->arena_bytes;
    srv->th = std::thread(scheduler, srv);
    if (prev >= 0) cudaSetDevice(prev);
    *out = srv;
    return LVBH_OK;
}

void lvbh_server_destroy(lvbh_server *srv) {
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
    }
    srv->cv.notify_all();
    if (srv->th.joinable()) srv->th.join();
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(srv->device);
    destroy_slots(srv);
    if (srv->arena) cudaFree(srv->arena);
    std::vector<Block *> blocks;
    for (auto &kv : srv->reqs) {
        Block *b = kv.second->block;
        if (b && std::find(blocks.begin(), blocks.end(), b) == blocks.end()) blocks.push_back(b);
        delete kv.second;
    }
    for (Block *b : blocks) delete b;
    cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    delete srv;
}

int lvbh_submit(lvbh_server *srv, const float *tri, uint32_t num_tris, const float *model_bounds,
                uint32_t flags, uint64_t *ticket) {
    if (!srv || !ticket) return LVBH_EINVAL;
    if (num_tris && !tri) return LVBH_EINVAL;
    if (num_tris > srv->max_tris) {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->err = "request larger than max_batch_tris";
        return LVBH_EINVAL;
    }
    if (num_tris && !(flags & LVBH_INPUT_HOST) && (reinterpret_cast<uintptr_t>(tri) & 15u)) {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->err = "device triangles must be 16-byte aligned";
        return LVBH_EINVAL;
    }
    if (BlockLayout(num_tris).bytes > srv->arena_bytes) {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->err = "request can never fit the result memory";
        return LVBH_ENOMEM;
    }
    Req *r = new (std::nothrow) Req();
    if (!r) return LVBH_ENOMEM;
    r->tri = tri;
    r->n = num_tris;
    r->host = (flags & LVBH_INPUT_HOST) != 0;
    if (model_bounds) {
        r->has_bounds = true;
        std::memcpy(r->bounds, model_bounds, sizeof r->bounds);
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (srv->stop || srv->reqs.size() >= srv->max_requests) {
            srv->err = srv->stop ? "server is stopping" : "too many requests held";
            delete r;
            return LVBH_EBUSY;
        }
        r->id = srv->next_id++;
        srv->reqs[r->id] = r;
        ++srv->st.submitted;
        if (num_tris == 0) {  // nothing to build: an empty result, as build() gives for NUM_TRIS 0
            r->status = LVBH_OK;
            r->t_launch = r->t_done = r->t_submit;
            if (model_bounds) std::memcpy(r->out_bounds, model_bounds, sizeof r->out_bounds);
            ++srv->st.completed;
        } else {
            srv->queue.push_back(r);
        }
        *ticket = r->id;
    }
    srv->cv.notify_all();
    return LVBH_OK;
}

int lvbh_poll(lvbh_server *srv, uint64_t ticket, lvbh_result *out, lvbh_request_info *info) {
    if (!srv) return LVBH_EINVAL;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(ticket);
    if (it == srv->reqs.end()) return LVBH_EINVAL;
    fill(srv, it->second, out, info);
    return it->second->status;
}

int lvbh_wait(lvbh_server *srv, uint64_t ticket, int timeout_ms, lvbh_result *out,
              lvbh_request_info *info) {
    if (!srv) return LVBH_EINVAL;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->reqs.find(ticket);
    if (it == srv->reqs.end()) return LVBH_EINVAL;
    Req *r = it->second;
    auto ready = [&] { return r->status != LVBH_EBUSY; };
    if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
    else srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    fill(srv, r, out, info);
    return r->status;
}

int lvbh_request_release(lvbh_server *srv, uint64_t ticket) {
    if (!srv) return LVBH_EINVAL;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        auto it = srv->reqs.find(ticket);
        if (it == srv->reqs.end()) return LVBH_EINVAL;
        Req *r = it->second;
        if (r->status == LVBH_EBUSY) return LVBH_EBUSY;
        if (Block *b = r->block) {
            if (--b->refs == 0) {
                srv->alloc.release(b->off, b->bytes);
                srv->mem_blocked = false;
                delete b;
            }
        }
        srv->reqs.erase(it);
        delete r;
    }
    srv->cv.notify_all();
    return LVBH_OK;
}

int lvbh_server_stats_get(lvbh_server *srv, lvbh_server_stats *out) {
    if (!srv || !out) return LVBH_EINVAL;
    std::lock_guard<std::mutex> lk(srv->mu);
    *out = srv->st;
    out->bytes_in_use = srv->alloc.used();
    out->peak_bytes = srv->alloc.peak();
    return LVBH_OK;
}

const char *lvbh_server_last_error(const lvbh_server *srv) {
    if (!srv) return "no server";
    return srv->err.c_str();
}

}  // extern "C"
