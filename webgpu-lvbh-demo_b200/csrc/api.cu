// api.cu - the C ABI (include/lvbh.h): context, scratch arena, build orchestration.
//
// Replaces the reference's host orchestration (scripts/bvh/build-bvh.js:12-66 and each kernel
// module's execute(): 69 queue submits and 20 host waits per build) with one stream-ordered
// chain of 8 kernels and a memset, replayed as a cached CUDA graph when the same build shape
// repeats, and a single host wait at the end (none with LVBH_ASYNC).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>

#include "lvbh.h"
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int v = 148;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) v = 148;
        cached[dev] = v;
    }
    return cached[dev];
}

}  // namespace lvbh

using namespace lvbh;

namespace {

constexpr size_t kAlign = 256;
// A host soup whose box is reduced on the device is uploaded in up to kUploadChunks chunks of
// at least kUploadChunkTris triangles (a multiple of the sort tile); each chunk's box and
// centroid pass runs on the build stream while the next chunk is copied.
constexpr uint32_t kUploadChunks = 8;
constexpr uint32_t kUploadChunkTris = 1u << 20;
inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// The head of the control block (test words, error words, tile counters, reduced bounds) is
// read back with each build into a 64-byte pinned buffer.
static_assert(offsetof(Control, pad1) <= 64, "control block head fits the pinned readback");

// The control block and the sort's tile / chunk histograms.
size_t control_bytes(uint32_t n) {
    return align_up(sizeof(Control)) + sort_scratch_words(n) * sizeof(uint32_t);
}

// Scratch of a context sized for `cap` triangles: sort ping-pong keys and values, the tree
// pass's open-node buffers, the control block and the look-back words.
size_t arena_bytes(uint32_t cap) {
    const size_t groups = emit_groups(cap);
    return 4 * align_up((size_t)cap * 4) + align_up((size_t)cap * 12) + align_up((size_t)cap * 32) + align_up((size_t)cap) +
           align_up(groups * kOpenCap * sizeof(OpenItem)) + align_up(groups * sizeof(uint32_t)) +
           align_up(sizeof(uint32_t)) + control_bytes(cap);
}

struct GraphKey {
    const void *tri = nullptr;
    const void *verts = nullptr, *idx3 = nullptr;  // mesh input (the indexed leaf format)
    uint32_t nverts = 0;
    uint32_t n = 0;
    HostBounds hb{};
    int pre = 0;
    void *outs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    bool operator==(const GraphKey &o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

// Tunables of a batched build and the histogram key the tuner caches them under: per
// power-of-two size class of the meshes, the bit length of the number of meshes in it.
struct Tunables {
    int digit_bits = kDigitBits;
    int log_block = kLogEmitBlock;
    int tree_ctas = 0;
};
struct TuneKey {
    uint8_t cls[33] = {};
    bool operator<(const TuneKey &o) const { return std::memcmp(cls, o.cls, sizeof cls) < 0; }
};
struct Tuned {
    Tunables t;
    float ms[4] = {0.f, 0.f, 0.f, 0.f};  // the candidates' times (0 = not timed)
    uint32_t candidates = 0;
};
constexpr Tunables kCandidates[4] = {{kDigitBits, 8, 0}, {kDigitBits, 7, 0}, {kDigitBits32, 8, 0},
                                     {kDigitBits32, 7, 0}};

struct BatchKey {
    const void *tri = nullptr;
    uint32_t total = 0, num_segs = 0, tiles = 0, blocks = 0, groups = 0;
    int use_bounds = 0, digit_bits = 0, log_block = 0, tree_ctas = 0;
    void *outs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    bool operator==(const BatchKey &o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

}  // namespace

struct lvbh_ctx {
    int device = 0;
    std::string err;
    // scratch arena (sized for `cap` triangles)
    uint32_t cap = 0;
    void *arena = nullptr;
    uint32_t *keys_b = nullptr, *vals_b = nullptr;
    uint32_t *keys_a = nullptr;  // unsorted Morton keys (input of the first sort pass)
    float *cen = nullptr;        // triangle centroids, x / y / z arrays of `cap` floats
    OpenItem *items = nullptr;
    uint32_t *counts = nullptr, *arrive = nullptr, *epoch = nullptr;
    float4 *pend = nullptr;
    uint8_t *pend_d = nullptr;
    Control *ctl = nullptr;
    uint32_t *lookback = nullptr;  // the sort's tile and chunk histograms
    // staging for host input
    size_t stage_bytes = 0;
    void *stage = nullptr;
    // pinned readback of the control block head
    uint32_t *host_ctl = nullptr;
    // the control block's test words (lvbh_test_stall_lookback), restored when the arena moves
    uint32_t test_stall1 = 0, test_spin = 0;
    uint32_t *trace_counter = nullptr;  // ray counter of the persistent traversal
    ObjScratch obj;                     // OBJ ingest buffers (the parsed soup among them)
    cudaEvent_t ev[LVBH_NUM_STAGES + 1] = {};
    bool ev_valid = false;
    // chunked upload of a host soup: its copy stream and events (start, one per chunk)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t up_ev[1 + kUploadChunks] = {};
    // cached graph of the last build shape
    cudaStream_t cap_stream = nullptr;
    GraphKey gkey;
    cudaGraphExec_t gexec = nullptr;
    // batched builds: segment table, per-segment bounds and histograms, look-back words and
    // open items (device), and a pinned mirror of the table, host bounds and reduced bounds
    uint32_t b_segs = 0, b_tiles = 0, b_blocks = 0;  // capacity
    void *b_dev = nullptr;
    SegRow *b_rows = nullptr;
    uint32_t *b_tile_seg = nullptr, *b_blk_seg = nullptr, *b_grp_seg = nullptr;
    uint32_t *b_zero = nullptr;  // seg_ord, seg_hist and look-back words, zeroed per build
    size_t b_zero_bytes = 0;
    uint32_t *b_ord = nullptr, *b_hist = nullptr, *b_lookback = nullptr;
    float *b_bounds = nullptr;
    OpenItem *b_items = nullptr;
    uint32_t *b_counts = nullptr;
    void *b_host = nullptr;
    SegRow *bh_rows = nullptr;
    float *bh_bounds = nullptr;
    uint32_t *bh_ord = nullptr;
    BatchKey bkey;
    cudaGraphExec_t bgexec = nullptr;
    // batched-build tunables: forced by the caller, or tuned per segment-size histogram
    bool forced = false;
    Tunables forced_t;
    std::map<TuneKey, Tuned> tuned;
    Tuned last_tuned;
    // last build, for lvbh_sync
    cudaStream_t last_stream = nullptr;
    lvbh_result *last_out = nullptr;
    HostBounds last_hb{};
    bool pending = false;
    bool last_batch = false;
    uint32_t last_segs = 0;
    float *last_bounds_out = nullptr;
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int fail(lvbh_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(lvbh_ctx *ctx, cudaError_t e, const char *what) {
    const int code = (e == cudaErrorMemoryAllocation) ? LVBH_ENOMEM : LVBH_ECUDA;
    cudaGetLastError();  // clear the sticky-free error state
    return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define LVBH_CUDA(ctx, call)                                              \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #call);        \
    } while (0)

void free_arena(lvbh_ctx *ctx) {
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    if (ctx->bgexec) { cudaGraphExecDestroy(ctx->bgexec); ctx->bgexec = nullptr; }
    if (ctx->arena) cudaFree(ctx->arena);
    ctx->arena = nullptr;
    ctx->cap = 0;
}

void free_batch(lvbh_ctx *ctx) {
    if (ctx->bgexec) { cudaGraphExecDestroy(ctx->bgexec); ctx->bgexec = nullptr; }
    if (ctx->b_dev) cudaFree(ctx->b_dev);
    if (ctx->b_host) cudaFreeHost(ctx->b_host);
    ctx->b_dev = ctx->b_host = nullptr;
    ctx->b_segs = ctx->b_tiles = ctx->b_blocks = 0;
}

// Device bytes of the batch scratch for `segs` segments, `tiles` sort tiles and `blocks` tree
// blocks: segment rows, tile / block / group -> segment maps, bounds, digit counts and
// look-back words, given bounds, open items and their per-block counts.
size_t batch_bytes(uint32_t segs, uint32_t tiles, uint32_t blocks) {
    const size_t rows = align_up((segs + 1ull) * sizeof(SegRow));
    const size_t ord = (size_t)segs * 6 * 4, hist = (size_t)segs * kHistWords * 4;
    const size_t lb = (size_t)kSortPasses * tiles * kDigits * 4;
    return rows + align_up(tiles * 4ull) + 2 * align_up(blocks * 4ull) + align_up(ord + hist + lb) +
           align_up((size_t)segs * 6 * 4) + align_up((size_t)blocks * kOpenCap * sizeof(OpenItem)) +
           align_up(blocks * 4ull);
}

// Batch scratch for up to `segs` segments, `tiles` sort tiles and `blocks` tree blocks.
int ensure_batch(lvbh_ctx *ctx, uint32_t segs, uint32_t tiles, uint32_t blocks) {
    if (ctx->b_dev && segs <= ctx->b_segs && tiles <= ctx->b_tiles && blocks <= ctx->b_blocks)
        return LVBH_OK;
    if (ctx->pending) cudaStreamSynchronize(ctx->last_stream);
    segs = segs > ctx->b_segs ? segs : ctx->b_segs;
    tiles = tiles > ctx->b_tiles ? tiles : ctx->b_tiles;
    blocks = blocks > ctx->b_blocks ? blocks : ctx->b_blocks;
    free_batch(ctx);
    const size_t rows = align_up((segs + 1ull) * sizeof(SegRow));
    const size_t ord = (size_t)segs * 6 * 4, hist = (size_t)segs * kHistWords * 4;
    const size_t lb = (size_t)kSortPasses * tiles * kDigits * 4;
    const size_t zero = align_up(ord + hist + lb);
    const size_t bnd = align_up((size_t)segs * 6 * 4);
    const size_t dev = batch_bytes(segs, tiles, blocks);
    void *p = nullptr;
    LVBH_CUDA(ctx, cudaMalloc(&p, dev));
    void *h = nullptr;
    const size_t host = rows + bnd + align_up(ord);
    cudaError_t e = cudaMallocHost(&h, host);
    if (e != cudaSuccess) { cudaFree(p); return cuda_fail(ctx, e, "cudaMallocHost(batch)"); }
    char *c = static_cast<char *>(p);
    ctx->b_dev = p;
    ctx->b_rows = reinterpret_cast<SegRow *>(c); c += rows;
    ctx->b_tile_seg = reinterpret_cast<uint32_t *>(c); c += align_up(tiles * 4ull);
    ctx->b_blk_seg = reinterpret_cast<uint32_t *>(c); c += align_up(blocks * 4ull);
    ctx->b_grp_seg = reinterpret_cast<uint32_t *>(c); c += align_up(blocks * 4ull);  // groups <= blocks
    ctx->b_zero = reinterpret_cast<uint32_t *>(c);
    ctx->b_ord = ctx->b_zero;
    ctx->b_hist = ctx->b_ord + (size_t)segs * 6;
    ctx->b_lookback = ctx->b_hist + (size_t)segs * kHistWords;
    c += zero;
    ctx->b_bounds = reinterpret_cast<float *>(c); c += bnd;
    ctx->b_items = reinterpret_cast<OpenItem *>(c); c += align_up((size_t)blocks * kOpenCap * sizeof(OpenItem));
    ctx->b_counts = reinterpret_cast<uint32_t *>(c);  // open items per tree block
    char *hc = static_cast<char *>(h);
    ctx->b_host = h;
    ctx->bh_rows = reinterpret_cast<SegRow *>(hc); hc += rows;
    ctx->bh_bounds = reinterpret_cast<float *>(hc); hc += bnd;
    ctx->bh_ord = reinterpret_cast<uint32_t *>(hc);
    ctx->b_segs = segs;
    ctx->b_tiles = tiles;
    ctx->b_blocks = blocks;
    return LVBH_OK;
}

int ensure_arena(lvbh_ctx *ctx, uint32_t n) {
    if (n <= ctx->cap && ctx->arena) return LVBH_OK;
    if (ctx->pending) cudaStreamSynchronize(ctx->last_stream);
    free_arena(ctx);
    // a multiple of 4: the centroid runs (stride cap) start on 16-byte boundaries
    const uint32_t cap = n < 4096 ? 4096 : (n + 3u) & ~3u;
    void *p = nullptr;
    LVBH_CUDA(ctx, cudaMalloc(&p, arena_bytes(cap)));
    char *c = static_cast<char *>(p);
    ctx->arena = p;
    const size_t kb = align_up((size_t)cap * 4);
    const size_t groups = emit_groups(cap);
    ctx->keys_b = reinterpret_cast<uint32_t *>(c); c += kb;
    ctx->vals_b = reinterpret_cast<uint32_t *>(c); c += kb;
    ctx->arrive = reinterpret_cast<uint32_t *>(c); c += kb;
    ctx->keys_a = reinterpret_cast<uint32_t *>(c); c += kb;
    ctx->cen = reinterpret_cast<float *>(c); c += align_up((size_t)cap * 12);
    ctx->pend = reinterpret_cast<float4 *>(c); c += align_up((size_t)cap * 32);
    ctx->pend_d = reinterpret_cast<uint8_t *>(c); c += align_up((size_t)cap);
    ctx->items = reinterpret_cast<OpenItem *>(c); c += align_up(groups * kOpenCap * sizeof(OpenItem));
    ctx->counts = reinterpret_cast<uint32_t *>(c); c += align_up(groups * sizeof(uint32_t));  // per tree block
    ctx->epoch = reinterpret_cast<uint32_t *>(c); c += align_up(sizeof(uint32_t));
    ctx->ctl = reinterpret_cast<Control *>(c);
    ctx->lookback = reinterpret_cast<uint32_t *>(c + align_up(sizeof(Control)));
    // arrival words and the epoch start at zero; from then on the epoch keeps them valid
    LVBH_CUDA(ctx, cudaMemset(ctx->arrive, 0, kb));
    LVBH_CUDA(ctx, cudaMemset(ctx->epoch, 0, sizeof(uint32_t)));
    // the control block's test words (zero unless lvbh_test_stall_lookback set them)
    const uint32_t test_words[2] = {ctx->test_stall1, ctx->test_spin};
    LVBH_CUDA(ctx, cudaMemcpy(ctx->ctl, test_words, sizeof test_words, cudaMemcpyHostToDevice));
    ctx->cap = cap;
    return LVBH_OK;
}

int ensure_stage(lvbh_ctx *ctx, size_t bytes) {
    if (bytes <= ctx->stage_bytes && ctx->stage) return LVBH_OK;
    if (ctx->pending) cudaStreamSynchronize(ctx->last_stream);
    if (ctx->stage) cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    if (ctx->bgexec) { cudaGraphExecDestroy(ctx->bgexec); ctx->bgexec = nullptr; }
    LVBH_CUDA(ctx, cudaMalloc(&ctx->stage, bytes));
    ctx->stage_bytes = bytes;
    return LVBH_OK;
}

// The build proper: every launch on `s`, nothing synchronous.
// A mesh input of the indexed leaf format: 16-byte vertex rows and index triples (device).
struct MeshIn {
    const float4 *verts;
    uint32_t nverts;
    const uint32_t *idx3;
};

// What upload_chunked did already, chunk by chunk behind the soup's upload (the control block
// is then cleared too): nothing, the box and centroids (no host bounds), or the keys (host
// bounds).
enum Pre : int { kPreNone = 0, kPreCen = 1, kPreKeys = 2 };

// An error: a launch could not be made (the tree pass's tensor map); the rest was enqueued.
cudaError_t enqueue_build(lvbh_ctx *ctx, const float4 *tri, uint32_t n, const HostBounds &hb,
                          const lvbh_result *out, cudaStream_t s, bool profile, const MeshIn *mesh = nullptr,
                          int pre = kPreNone) {
    if (profile) cudaEventRecord(ctx->ev[1], s);
    if (pre == kPreNone)
        cudaMemsetAsync(reinterpret_cast<char *>(ctx->ctl) + offsetof(Control, err), 0,
                        sizeof(Control) - offsetof(Control, err), s);
    // a soup whose box is reduced here: box and centroids in one pass, then the keys from the
    // centroids
    const bool cen_path = !hb.use && !mesh;
    if (!hb.use && pre == kPreNone) {
        if (mesh) launch_bounds_mesh(mesh->verts, mesh->nverts, mesh->idx3, n, ctx->ctl, s);
        else launch_bounds_cen(tri, 0, n, ctx->cen, ctx->cap, ctx->ctl, s);
    }
    if (profile) cudaEventRecord(ctx->ev[2], s);
    // unsorted keys go to keys_a, so that the three passes ping-pong keys_a -> result ->
    // scratch -> result
    uint32_t *keys_a = ctx->keys_a;
    if (mesh) launch_morton_mesh(mesh->verts, mesh->nverts, mesh->idx3, n, hb, ctx->ctl, keys_a, ctx->epoch,
                                 ctx->lookback, s);
    else if (cen_path) launch_morton_cen(ctx->cen, ctx->cap, n, ctx->ctl, keys_a, ctx->epoch, ctx->lookback, s);
    else if (pre != kPreKeys) launch_morton(tri, n, hb, ctx->ctl, keys_a, ctx->epoch, ctx->lookback, s);
    if (profile) cudaEventRecord(ctx->ev[3], s);
    launch_sort_pass(keys_a, nullptr, out->morton, out->leaf_index, n, 0, true, ctx->ctl, ctx->lookback, s);
    launch_sort_pass(out->morton, out->leaf_index, ctx->keys_b, ctx->vals_b, n, 1, false, ctx->ctl, ctx->lookback, s);
    launch_sort_pass(ctx->keys_b, ctx->vals_b, out->morton, out->leaf_index, n, 2, false, ctx->ctl, ctx->lookback, s);
    if (profile) cudaEventRecord(ctx->ev[4], s);
    if (mesh) {
        uint32_t *sidx = static_cast<uint32_t *>(out->tris);
        launch_leaf_idx(mesh->idx3, out->leaf_index, n, sidx, s);
        launch_emit_mesh(mesh->verts, mesh->nverts, sidx, out->morton, n, static_cast<float4 *>(out->nodes),
                         out->parents, ctx->items, ctx->counts, ctx->arrive, ctx->pend, ctx->pend_d, ctx->epoch,
                         ctx->ctl, s, profile ? ctx->ev + 5 : nullptr);
        return cudaSuccess;
    }
    return launch_emit(tri, out->leaf_index, out->morton, n, static_cast<float4 *>(out->tris),
                       static_cast<float4 *>(out->nodes), out->parents, ctx->items, ctx->counts,
                       ctx->arrive, ctx->pend, ctx->pend_d, ctx->epoch, ctx->ctl, s,
                       profile ? ctx->ev + 5 : nullptr);
}

// The batched build: every launch on `s`.  The segment table (and host bounds) are copied from
// the pinned mirror, so a replayed graph picks up the table of the current call.
cudaError_t enqueue_batch(lvbh_ctx *ctx, const float4 *tri, const BatchPlan &bp, bool use_bounds,
                          const lvbh_result *out, cudaStream_t s, bool profile) {
    if (profile) cudaEventRecord(ctx->ev[1], s);
    cudaMemcpyAsync(ctx->b_rows, ctx->bh_rows, (bp.num_segs + 1ull) * sizeof(SegRow),
                    cudaMemcpyHostToDevice, s);
    if (use_bounds)
        cudaMemcpyAsync(ctx->b_bounds, ctx->bh_bounds, bp.num_segs * 6ull * sizeof(float),
                        cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(reinterpret_cast<char *>(ctx->ctl) + offsetof(Control, err), 0,
                    sizeof(Control) - offsetof(Control, err), s);
    const bool wide = bp.digit_bits == kDigitBits;
    const size_t lb_words = wide ? (size_t)kSortPasses * kDigits : (size_t)kSortPasses32 * kDigits32;
    const uint32_t *zero_end = ctx->b_lookback + lb_words * bp.tiles;
    cudaMemsetAsync(ctx->b_zero, 0, (zero_end - ctx->b_zero) * sizeof(uint32_t), s);
    launch_seg_tables(ctx->b_rows, bp.num_segs, ctx->b_tile_seg, ctx->b_blk_seg, ctx->b_grp_seg, s);
    launch_bounds_batch(bp, tri, use_bounds ? ctx->b_bounds : nullptr, ctx->b_ord, s);
    if (profile) cudaEventRecord(ctx->ev[2], s);
    uint32_t *keys_a = ctx->keys_a;
    launch_morton_batch(bp, tri, use_bounds ? ctx->b_bounds : nullptr, ctx->b_ord, ctx->b_hist,
                        ctx->ctl, keys_a, ctx->epoch, s);
    if (profile) cudaEventRecord(ctx->ev[3], s);
    // ping-pong so that the last pass lands in the result buffers
    uint32_t *kb = ctx->keys_b, *vb = ctx->vals_b, *ko = out->morton, *vo = out->leaf_index;
    if (wide) {
        launch_onesweep_batch(bp, keys_a, nullptr, ko, vo, 0, ctx->b_hist, ctx->ctl, ctx->b_lookback, s);
        launch_onesweep_batch(bp, ko, vo, kb, vb, 1, ctx->b_hist, ctx->ctl, ctx->b_lookback, s);
        launch_onesweep_batch(bp, kb, vb, ko, vo, 2, ctx->b_hist, ctx->ctl, ctx->b_lookback, s);
    } else {
        launch_onesweep_batch(bp, keys_a, nullptr, kb, vb, 0, ctx->b_hist, ctx->ctl, ctx->b_lookback, s);
        launch_onesweep_batch(bp, kb, vb, ko, vo, 1, ctx->b_hist, ctx->ctl, ctx->b_lookback, s);
        launch_onesweep_batch(bp, ko, vo, kb, vb, 2, ctx->b_hist, ctx->ctl, ctx->b_lookback, s);
        launch_onesweep_batch(bp, kb, vb, ko, vo, 3, ctx->b_hist, ctx->ctl, ctx->b_lookback, s);
    }
    if (profile) cudaEventRecord(ctx->ev[4], s);
    return launch_emit_batch(bp, tri, out->leaf_index, out->morton, static_cast<float4 *>(out->tris),
                             static_cast<float4 *>(out->nodes), out->parents, ctx->b_items,
                             ctx->b_counts, ctx->arrive, ctx->pend, ctx->pend_d, ctx->epoch, ctx->ctl, s,
                             profile ? ctx->ev + 5 : nullptr);
}

int launch_batch_graph(lvbh_ctx *ctx, const float4 *tri, const BatchPlan &bp, bool use_bounds,
                       const lvbh_result *out, cudaStream_t s) {
    BatchKey key;
    std::memset(static_cast<void *>(&key), 0, sizeof key);
    key.tri = tri;
    key.total = bp.total;
    key.num_segs = bp.num_segs;
    key.tiles = bp.tiles;
    key.blocks = bp.blocks;
    key.groups = bp.groups;  // the straddling pass's grid
    key.use_bounds = use_bounds;
    key.digit_bits = bp.digit_bits;
    key.log_block = bp.log_block;
    key.tree_ctas = bp.tree_ctas_per_sm;
    key.outs[0] = out->nodes; key.outs[1] = out->tris; key.outs[2] = out->parents;
    key.outs[3] = out->leaf_index; key.outs[4] = out->morton;
    if (!ctx->bgexec || !(key == ctx->bkey)) {
        if (ctx->bgexec) { cudaGraphExecDestroy(ctx->bgexec); ctx->bgexec = nullptr; }
        if (!ctx->cap_stream) LVBH_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
        LVBH_CUDA(ctx, cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t qe = enqueue_batch(ctx, tri, bp, use_bounds, out, ctx->cap_stream, false);
        cudaGraph_t g = nullptr;
        LVBH_CUDA(ctx, cudaStreamEndCapture(ctx->cap_stream, &g));
        if (qe != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(ctx, qe, "tree pass tensor map"); }
        cudaError_t e = cudaGraphInstantiate(&ctx->bgexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { ctx->bgexec = nullptr; return cuda_fail(ctx, e, "cudaGraphInstantiate(batch)"); }
        ctx->bkey = key;
    }
    LVBH_CUDA(ctx, cudaGraphLaunch(ctx->bgexec, s));
    return LVBH_OK;
}

int launch_graph(lvbh_ctx *ctx, const float4 *tri, uint32_t n, const HostBounds &hb,
                 const lvbh_result *out, cudaStream_t s, const MeshIn *mesh, int pre) {
    GraphKey key;
    std::memset(static_cast<void *>(&key), 0, sizeof key);  // padding takes part in the compare
    key.tri = tri;
    if (mesh) {
        key.verts = mesh->verts;
        key.idx3 = mesh->idx3;
        key.nverts = mesh->nverts;
    }
    key.n = n;
    key.hb = hb;
    key.pre = pre;
    key.outs[0] = out->nodes; key.outs[1] = out->tris; key.outs[2] = out->parents;
    key.outs[3] = out->leaf_index; key.outs[4] = out->morton;
    if (!ctx->gexec || !(key == ctx->gkey)) {
        if (!ctx->cap_stream) LVBH_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
        LVBH_CUDA(ctx, cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t qe = enqueue_build(ctx, tri, n, hb, out, ctx->cap_stream, false, mesh, pre);
        cudaGraph_t g = nullptr;
        LVBH_CUDA(ctx, cudaStreamEndCapture(ctx->cap_stream, &g));
        if (qe != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(ctx, qe, "tree pass tensor map"); }
        bool updated = false;
        if (ctx->gexec) {
            cudaGraphExecUpdateResultInfo info;
            updated = cudaGraphExecUpdate(ctx->gexec, g, &info) == cudaSuccess;
            if (!updated) {
                cudaGetLastError();
                cudaGraphExecDestroy(ctx->gexec);
                ctx->gexec = nullptr;
            }
        }
        cudaError_t e = cudaSuccess;
        if (!updated) e = cudaGraphInstantiate(&ctx->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) { ctx->gexec = nullptr; return cuda_fail(ctx, e, "cudaGraphInstantiate"); }
        ctx->gkey = key;
    }
    LVBH_CUDA(ctx, cudaGraphLaunch(ctx->gexec, s));
    return LVBH_OK;
}

int alloc_outputs(lvbh_ctx *ctx, uint32_t n, lvbh_result *out, size_t tri_row = 48) {
    out->nodes = out->tris = nullptr;
    out->parents = nullptr;
    out->leaf_index = out->morton = nullptr;
    out->owned = 0;
    if (n == 0) return LVBH_OK;
    void *p[5] = {};
    const size_t sz[5] = {64ull * n, tri_row * n, 8ull * n, 4ull * n, 4ull * n};
    for (int i = 0; i < 5; ++i) {
        cudaError_t e = cudaMalloc(&p[i], sz[i]);
        if (e != cudaSuccess) {
            for (int j = 0; j < i; ++j) cudaFree(p[j]);
            return cuda_fail(ctx, e, "cudaMalloc(result)");
        }
    }
    out->nodes = p[0];
    out->tris = p[1];
    out->parents = static_cast<int32_t *>(p[2]);
    out->leaf_index = static_cast<uint32_t *>(p[3]);
    out->morton = static_cast<uint32_t *>(p[4]);
    out->owned = 1;
    return LVBH_OK;
}

int build_common(lvbh_ctx *ctx, const float4 *tri_dev, uint32_t n, const float *model_bounds,
                 uint32_t flags, lvbh_result *out, cudaStream_t s, bool profile_upload,
                 const MeshIn *mesh = nullptr, int pre = kPreNone) {
    HostBounds hb{};
    if (model_bounds) {
        std::memcpy(hb.v, model_bounds, sizeof hb.v);
        hb.use = 1;
    }
    const bool profile = (flags & LVBH_PROFILE) != 0;
    if (n == 0) {
        ctx->pending = false;
        ctx->ev_valid = false;
        if (model_bounds) std::memcpy(out->bounds, model_bounds, sizeof out->bounds);
        return LVBH_OK;
    }
    int rc = LVBH_OK;
    if (profile && !profile_upload) cudaEventRecord(ctx->ev[0], s);
    if (profile || (flags & LVBH_NO_GRAPH)) {
        const cudaError_t qe = enqueue_build(ctx, tri_dev, n, hb, out, s, profile, mesh, pre);
        cudaError_t e = cudaGetLastError();
        if (qe != cudaSuccess) return cuda_fail(ctx, qe, "tree pass tensor map");
        if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
    } else {
        rc = launch_graph(ctx, tri_dev, n, hb, out, s, mesh, pre);
        if (rc) return rc;
    }
    ctx->ev_valid = profile;
    // fetch the error words and the device-reduced bounds with the build
    LVBH_CUDA(ctx, cudaMemcpyAsync(ctx->host_ctl, ctx->ctl, offsetof(Control, pad1),
                                   cudaMemcpyDeviceToHost, s));
    ctx->last_stream = s;
    ctx->last_out = out;
    ctx->last_hb = hb;
    ctx->last_batch = false;
    ctx->pending = true;
    if (flags & LVBH_ASYNC) return LVBH_OK;
    return lvbh_sync(ctx);
}

// Host inverse of the device's order-preserving float -> uint32 map (ord_lo).
float ord_word_to_float(uint32_t o) {
    const uint32_t u = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

int check_out(lvbh_ctx *ctx, uint32_t n, uint32_t flags, lvbh_result *out, size_t tri_row = 48) {
    if (!out) return fail(ctx, LVBH_EINVAL, "out is NULL");
    if (flags & LVBH_OUT_CALLER) {
        if (n && (!out->nodes || !out->tris || !out->parents || !out->leaf_index || !out->morton))
            return fail(ctx, LVBH_EINVAL, "LVBH_OUT_CALLER with a NULL result buffer");
        if (n && (((uintptr_t)out->nodes | (tri_row == 48 ? (uintptr_t)out->tris : 0)) & 15u))
            return fail(ctx, LVBH_EINVAL, "result nodes/tris must be 16-byte aligned");
        if (n && ((uintptr_t)out->tris & 3u))
            return fail(ctx, LVBH_EINVAL, "result tris must be 4-byte aligned");
        if (n && (((uintptr_t)out->parents | (uintptr_t)out->leaf_index | (uintptr_t)out->morton) & 3u))
            return fail(ctx, LVBH_EINVAL, "result parents/leaf_index/morton must be 4-byte aligned");
        out->owned = 0;
        return LVBH_OK;
    }
    return alloc_outputs(ctx, n, out, tri_row);
}

// A build entry first completes the context's pending LVBH_ASYNC build, before it touches
// any buffer that build may still use (arena, staging copy, pinned mirrors).  When the pending
// build failed, its status is returned and no new build starts, so the status is not lost.
// A host soup to the staging buffer in chunks on the context's copy stream; the build stream
// runs each chunk's first pass as soon as the chunk has landed, so that pass hides behind the
// upload: the box and centroid pass without host bounds, the Morton keys with them.  Clears
// the control block first (the build then skips its clear).  Returns the Pre the build goes on
// from.
int upload_chunked(lvbh_ctx *ctx, const float *host, uint32_t n, const float *model_bounds, cudaStream_t s,
                   int *pre) {
    if (!ctx->copy_stream) LVBH_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    for (auto &e : ctx->up_ev)
        if (!e) LVBH_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    LVBH_CUDA(ctx, cudaMemsetAsync(reinterpret_cast<char *>(ctx->ctl) + offsetof(Control, err), 0,
                                   sizeof(Control) - offsetof(Control, err), s));
    // the copies wait for earlier work on s (an earlier build may still read the staging buffer)
    LVBH_CUDA(ctx, cudaEventRecord(ctx->up_ev[0], s));
    LVBH_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->up_ev[0], 0));
    HostBounds hb{};
    if (model_bounds) {
        std::memcpy(hb.v, model_bounds, sizeof hb.v);
        hb.use = 1;
    }
    // chunks end on Morton-pass chunks of sort tiles (the key pass runs per chunk)
    const uint32_t unit = sort_chunk_tiles(n) * (uint32_t)kSortTile, units = sort_chunks(n);
    uint32_t chunks = n / kUploadChunkTris;
    if (chunks > kUploadChunks) chunks = kUploadChunks;
    if (chunks < 1) chunks = 1;
    const uint32_t per = (units + chunks - 1) / chunks;  // Morton chunks per upload chunk
    char *stage = static_cast<char *>(ctx->stage);
    const float4 *tri = static_cast<const float4 *>(ctx->stage);
    const char *src = reinterpret_cast<const char *>(host);
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t u0 = c * per, u1 = std::min(units, (c + 1) * per);
        if (u0 >= u1) break;
        const uint32_t t0 = u0 * unit, t1 = std::min(n, u1 * unit);
        LVBH_CUDA(ctx, cudaMemcpyAsync(stage + 48ull * t0, src + 48ull * t0, 48ull * (t1 - t0),
                                       cudaMemcpyHostToDevice, ctx->copy_stream));
        LVBH_CUDA(ctx, cudaEventRecord(ctx->up_ev[1 + c], ctx->copy_stream));
        LVBH_CUDA(ctx, cudaStreamWaitEvent(s, ctx->up_ev[1 + c], 0));
        if (hb.use) launch_morton_chunks(tri, n, hb, ctx->ctl, ctx->keys_a, ctx->epoch, ctx->lookback, u0, u1, s);
        else launch_bounds_cen(tri, t0, t1, ctx->cen, ctx->cap, ctx->ctl, s);
    }
    *pre = hb.use ? kPreKeys : kPreCen;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
    return LVBH_OK;
}

int finish_pending(lvbh_ctx *ctx) {
    if (!ctx->pending) return LVBH_OK;
    const int rc = lvbh_sync(ctx);
    if (rc != LVBH_OK) ctx->err = "an earlier LVBH_ASYNC build failed: " + ctx->err;
    return rc;
}

}  // namespace

namespace lvbh {

int ctx_reserve_batch(lvbh_ctx *ctx, uint32_t max_tris, uint32_t max_segs) {
    if (!ctx) return LVBH_EINVAL;
    DeviceGuard g(ctx->device);
    if (int rc = ensure_arena(ctx, max_tris)) return rc;
    return ensure_batch(ctx, max_segs, sort_tiles(max_tris) + max_segs,
                        (uint32_t)emit_groups(max_tris) + max_segs);
}

size_t ctx_device_bytes(const lvbh_ctx *ctx) {
    if (!ctx || !ctx->arena) return 0;
    const uint32_t segs = ctx->b_segs, tiles = ctx->b_tiles, blocks = ctx->b_blocks;
    size_t batch = 0;
    if (ctx->b_dev) batch = batch_bytes(segs, tiles, blocks);
    return arena_bytes(ctx->cap) + batch + ctx->stage_bytes;
}

}  // namespace lvbh

extern "C" {

const char *lvbh_version(void) { return "lvbh-b200 0.1 (sm_100a)"; }

int lvbh_create(lvbh_ctx **out, const lvbh_config *cfg) {
    if (!out) return LVBH_EINVAL;
    *out = nullptr;
    int dev = cfg ? cfg->device : -1;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return LVBH_ECUDA; }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || dev >= count) { cudaGetLastError(); return LVBH_EINVAL; }
    lvbh_ctx *ctx = new (std::nothrow) lvbh_ctx();
    if (!ctx) return LVBH_ENOMEM;
    ctx->device = dev;
    DeviceGuard g(dev);
    if (cudaMallocHost(&ctx->host_ctl, 64) != cudaSuccess) { cudaGetLastError(); delete ctx; return LVBH_ENOMEM; }
    for (auto &e : ctx->ev) {
        if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); lvbh_destroy(ctx); return LVBH_ECUDA; }
    }
    if (emit_init() != cudaSuccess || sort_init() != cudaSuccess || morton_init() != cudaSuccess) {
        cudaGetLastError();
        lvbh_destroy(ctx);
        return LVBH_ECUDA;
    }
    if (cfg && cfg->reserve_tris) {
        if (cfg->reserve_tris > LVBH_MAX_TRIS) { lvbh_destroy(ctx); return LVBH_EINVAL; }
        if (int rc = ensure_arena(ctx, cfg->reserve_tris)) { lvbh_destroy(ctx); return rc; }
    }
    *out = ctx;
    return LVBH_OK;
}

void lvbh_destroy(lvbh_ctx *ctx) {
    if (!ctx) return;
    DeviceGuard g(ctx->device);
    if (ctx->pending) cudaStreamSynchronize(ctx->last_stream);
    free_arena(ctx);
    free_batch(ctx);
    if (ctx->stage) cudaFree(ctx->stage);
    for (auto &e : ctx->ev) if (e) cudaEventDestroy(e);
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    for (auto &e : ctx->up_ev) if (e) cudaEventDestroy(e);
    if (ctx->host_ctl) cudaFreeHost(ctx->host_ctl);
    if (ctx->trace_counter) cudaFree(ctx->trace_counter);
    obj_free(ctx->obj);
    cudaGetLastError();
    delete ctx;
}

int lvbh_build_soup(lvbh_ctx *ctx, const float *tri_array, uint32_t num_tris,
                    const float *model_bounds, uint32_t flags, lvbh_result *out, void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (!out) return fail(ctx, LVBH_EINVAL, "out is NULL");
    if (num_tris > LVBH_MAX_TRIS) return fail(ctx, LVBH_EINVAL, "num_tris exceeds LVBH_MAX_TRIS");
    if (num_tris && !tri_array) return fail(ctx, LVBH_EINVAL, "tri_array is NULL");
    DeviceGuard g(ctx->device);
    if (int rc = finish_pending(ctx)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (int rc = check_out(ctx, num_tris, flags, out)) return rc;
    out->num_tris = out->num_nodes = num_tris;
    std::memset(out->bounds, 0, sizeof out->bounds);
    if (num_tris) {
        if (int rc = ensure_arena(ctx, num_tris)) return rc;
        LVBH_CUDA(ctx, cudaMemsetAsync(&ctx->ctl->aux_err, 0, sizeof(uint32_t), s));
    }
    const float4 *tri = reinterpret_cast<const float4 *>(tri_array);
    bool profile_upload = false;
    if ((flags & LVBH_INPUT_HOST) && num_tris) {
        if (int rc = ensure_stage(ctx, 48ull * num_tris)) return rc;
        if (!(flags & LVBH_PROFILE) && num_tris >= 2 * kUploadChunkTris) {
            int pre = kPreNone;
            if (int rc = upload_chunked(ctx, tri_array, num_tris, model_bounds, s, &pre)) return rc;
            return build_common(ctx, static_cast<const float4 *>(ctx->stage), num_tris, model_bounds, flags,
                                out, s, false, nullptr, pre);
        }
        if (flags & LVBH_PROFILE) { cudaEventRecord(ctx->ev[0], s); profile_upload = true; }
        LVBH_CUDA(ctx, cudaMemcpyAsync(ctx->stage, tri_array, 48ull * num_tris, cudaMemcpyHostToDevice, s));
        tri = static_cast<const float4 *>(ctx->stage);
    } else if (num_tris && (reinterpret_cast<uintptr_t>(tri_array) & 15u)) {
        return fail(ctx, LVBH_EINVAL, "device tri_array must be 16-byte aligned");
    }
    return build_common(ctx, tri, num_tris, model_bounds, flags, out, s, profile_upload);
}

int lvbh_build_indexed(lvbh_ctx *ctx, const float *xyz, uint32_t num_verts, const uint32_t *idx3,
                       uint32_t num_tris, const float *model_bounds, uint32_t flags,
                       lvbh_result *out, void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (!out) return fail(ctx, LVBH_EINVAL, "out is NULL");
    if (num_tris > LVBH_MAX_TRIS) return fail(ctx, LVBH_EINVAL, "num_tris exceeds LVBH_MAX_TRIS");
    if (num_tris && (!xyz || !idx3 || !num_verts)) return fail(ctx, LVBH_EINVAL, "NULL vertex or index buffer");
    DeviceGuard g(ctx->device);
    if (int rc = finish_pending(ctx)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (int rc = check_out(ctx, num_tris, flags, out)) return rc;
    out->num_tris = out->num_nodes = num_tris;
    std::memset(out->bounds, 0, sizeof out->bounds);
    if (!num_tris) return build_common(ctx, nullptr, 0, model_bounds, flags, out, s, false);
    if (flags & LVBH_INPUT_HOST) {
        // indices are validated on the host when they are host memory
        for (uint64_t i = 0; i < 3ull * num_tris; ++i)
            if (idx3[i] >= num_verts) return fail(ctx, LVBH_EINVAL, "vertex index out of range");
    }
    const size_t soup = align_up(48ull * num_tris);
    const size_t vb = align_up(12ull * num_verts), ib = align_up(12ull * num_tris);
    const bool host = (flags & LVBH_INPUT_HOST) != 0;
    if (int rc = ensure_arena(ctx, num_tris)) return rc;
    if (int rc = ensure_stage(ctx, soup + (host ? vb + ib : 0))) return rc;
    LVBH_CUDA(ctx, cudaMemsetAsync(&ctx->ctl->aux_err, 0, sizeof(uint32_t), s));
    char *st = static_cast<char *>(ctx->stage);
    bool profile_upload = false;
    if (flags & LVBH_PROFILE) { cudaEventRecord(ctx->ev[0], s); profile_upload = true; }
    if (host) {
        LVBH_CUDA(ctx, cudaMemcpyAsync(st + soup, xyz, 12ull * num_verts, cudaMemcpyHostToDevice, s));
        LVBH_CUDA(ctx, cudaMemcpyAsync(st + soup + vb, idx3, 12ull * num_tris, cudaMemcpyHostToDevice, s));
        xyz = reinterpret_cast<const float *>(st + soup);
        idx3 = reinterpret_cast<const uint32_t *>(st + soup + vb);
    }
    launch_gather_indexed(xyz, num_verts, idx3, num_tris, reinterpret_cast<float4 *>(st),
                          &ctx->ctl->aux_err, s);
    return build_common(ctx, reinterpret_cast<const float4 *>(st), num_tris, model_bounds, flags,
                        out, s, profile_upload);
}

int lvbh_build_mesh(lvbh_ctx *ctx, const float *verts4, uint32_t num_verts, const uint32_t *idx3,
                    uint32_t num_tris, const float *model_bounds, uint32_t flags, lvbh_result *out,
                    void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (!out) return fail(ctx, LVBH_EINVAL, "out is NULL");
    if (num_tris > LVBH_MAX_TRIS) return fail(ctx, LVBH_EINVAL, "num_tris exceeds LVBH_MAX_TRIS");
    if (num_tris && (!verts4 || !idx3 || !num_verts)) return fail(ctx, LVBH_EINVAL, "NULL vertex or index buffer");
    const bool host = (flags & LVBH_INPUT_HOST) != 0;
    if (num_tris && !host && ((reinterpret_cast<uintptr_t>(verts4) & 15u) || (reinterpret_cast<uintptr_t>(idx3) & 3u)))
        return fail(ctx, LVBH_EINVAL, "device vertex rows must be 16-byte aligned, indices 4-byte aligned");
    DeviceGuard g(ctx->device);
    if (int rc = finish_pending(ctx)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (int rc = check_out(ctx, num_tris, flags, out, 12)) return rc;
    out->num_tris = out->num_nodes = num_tris;
    std::memset(out->bounds, 0, sizeof out->bounds);
    if (!num_tris) return build_common(ctx, nullptr, 0, model_bounds, flags, out, s, false);
    if (int rc = ensure_arena(ctx, num_tris)) return rc;
    LVBH_CUDA(ctx, cudaMemsetAsync(&ctx->ctl->aux_err, 0, sizeof(uint32_t), s));
    bool profile_upload = false;
    if (host) {
        const size_t vb = align_up(16ull * num_verts), ib = align_up(12ull * num_tris);
        if (int rc = ensure_stage(ctx, vb + ib)) return rc;
        if (flags & LVBH_PROFILE) { cudaEventRecord(ctx->ev[0], s); profile_upload = true; }
        char *st = static_cast<char *>(ctx->stage);
        LVBH_CUDA(ctx, cudaMemcpyAsync(st, verts4, 16ull * num_verts, cudaMemcpyHostToDevice, s));
        LVBH_CUDA(ctx, cudaMemcpyAsync(st + vb, idx3, 12ull * num_tris, cudaMemcpyHostToDevice, s));
        verts4 = reinterpret_cast<const float *>(st);
        idx3 = reinterpret_cast<const uint32_t *>(st + vb);
    }
    const MeshIn mesh{reinterpret_cast<const float4 *>(verts4), num_verts, idx3};
    return build_common(ctx, nullptr, num_tris, model_bounds, flags, out, s, profile_upload, &mesh);
}

int lvbh_trace_mesh(lvbh_ctx *ctx, const void *nodes, const uint32_t *leaf_idx3, const float *verts4,
                    uint32_t num_verts, uint32_t num_tris, const float *rays, uint32_t num_rays,
                    int32_t *hit_prim, float *hit_t, uint32_t *max_stack, void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (num_rays && (!rays || !hit_prim || !hit_t)) return fail(ctx, LVBH_EINVAL, "NULL ray buffer");
    if (num_tris && (!nodes || !leaf_idx3 || !verts4 || !num_verts)) return fail(ctx, LVBH_EINVAL, "NULL tree buffer");
    DeviceGuard g(ctx->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!ctx->trace_counter) LVBH_CUDA(ctx, cudaMalloc(&ctx->trace_counter, sizeof(uint32_t)));
    launch_trace_mesh(static_cast<const float4 *>(nodes), reinterpret_cast<const float4 *>(verts4), num_verts,
                      leaf_idx3, num_tris, reinterpret_cast<const float4 *>(rays), num_rays, hit_prim, hit_t,
                      max_stack, ctx->trace_counter, s);
    LVBH_CUDA(ctx, cudaGetLastError());
    LVBH_CUDA(ctx, cudaStreamSynchronize(s));
    return LVBH_OK;
}

int lvbh_build_batched(lvbh_ctx *ctx, const float *tri_array, const uint32_t *seg_offsets,
                       uint32_t num_segs, const float *seg_bounds, float *bounds_out,
                       uint32_t flags, lvbh_result *out, void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (!out) return fail(ctx, LVBH_EINVAL, "out is NULL");
    if (num_segs && !seg_offsets) return fail(ctx, LVBH_EINVAL, "seg_offsets is NULL");
    if (num_segs > (1u << 24)) return fail(ctx, LVBH_EINVAL, "num_segs exceeds 2^24");
    if (num_segs && seg_offsets[0] != 0) return fail(ctx, LVBH_EINVAL, "seg_offsets[0] must be 0");
    uint64_t tiles = 0, blocks128 = 0;
    TuneKey tkey;
    for (uint32_t i = 0; i < num_segs; ++i) {
        if (seg_offsets[i + 1] < seg_offsets[i]) return fail(ctx, LVBH_EINVAL, "seg_offsets must be non-decreasing");
        const uint32_t n = seg_offsets[i + 1] - seg_offsets[i];
        tiles += sort_tiles(n);
        blocks128 += emit_groups(n, 7);
        const int c = n ? 32 - __builtin_clz(n) : 0;  // size class: bit length of n
        if (tkey.cls[c] < 255) ++tkey.cls[c];
    }
    for (uint8_t &v : tkey.cls) v = v ? (uint8_t)(32 - __builtin_clz(v)) : 0;
    const uint32_t total = num_segs ? seg_offsets[num_segs] : 0;
    if (total > LVBH_MAX_TRIS) return fail(ctx, LVBH_EINVAL, "total triangles exceed LVBH_MAX_TRIS");
    if (total && !tri_array) return fail(ctx, LVBH_EINVAL, "tri_array is NULL");
    DeviceGuard g(ctx->device);
    if (int rc = finish_pending(ctx)) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (int rc = check_out(ctx, total, flags, out)) return rc;
    out->num_tris = out->num_nodes = total;
    std::memset(out->bounds, 0, sizeof out->bounds);
    if (total == 0) {
        ctx->pending = false;
        ctx->ev_valid = false;
        for (uint64_t i = 0; bounds_out && i < num_segs * 6ull; ++i)
            bounds_out[i] = (seg_bounds && !std::isnan(seg_bounds[i - i % 6])) ? seg_bounds[i] : 0.0f;
        return LVBH_OK;
    }
    if (int rc = ensure_arena(ctx, total)) return rc;
    if (int rc = ensure_batch(ctx, num_segs, (uint32_t)tiles, (uint32_t)blocks128)) return rc;
    if (seg_bounds) std::memcpy(ctx->bh_bounds, seg_bounds, num_segs * 6ull * sizeof(float));
    // segment table for tree blocks of 2^log_block leaves: first triangle, first sort tile,
    // first tree block and first straddling-pass group (16 blocks of one segment) per segment
    auto plan = [&](const Tunables &t) {
        uint32_t tile = 0, blk = 0, grp = 0;
        for (uint32_t i = 0; i <= num_segs; ++i) {
            ctx->bh_rows[i] = SegRow{seg_offsets[i], tile, blk, grp};
            if (i < num_segs) {
                const uint32_t n = seg_offsets[i + 1] - seg_offsets[i];
                const uint32_t b = (uint32_t)emit_groups(n, t.log_block);
                tile += sort_tiles(n);
                blk += b;
                grp += straddle_groups(b);
            }
        }
        return BatchPlan{ctx->b_rows, ctx->b_tile_seg, ctx->b_blk_seg, ctx->b_grp_seg, num_segs,
                         (uint32_t)tiles, blk, total, grp, t.digit_bits, t.log_block, t.tree_ctas};
    };
    LVBH_CUDA(ctx, cudaMemsetAsync(&ctx->ctl->aux_err, 0, sizeof(uint32_t), s));
    const float4 *tri = reinterpret_cast<const float4 *>(tri_array);
    const bool profile = (flags & LVBH_PROFILE) != 0;
    if (profile) cudaEventRecord(ctx->ev[0], s);
    if (flags & LVBH_INPUT_HOST) {
        if (int rc = ensure_stage(ctx, 48ull * total)) return rc;
        LVBH_CUDA(ctx, cudaMemcpyAsync(ctx->stage, tri_array, 48ull * total, cudaMemcpyHostToDevice, s));
        tri = static_cast<const float4 *>(ctx->stage);
    } else if (reinterpret_cast<uintptr_t>(tri_array) & 15u) {
        return fail(ctx, LVBH_EINVAL, "device tri_array must be 16-byte aligned");
    }
    // the tunables: forced, tuned before for this size histogram, tuned now, or the defaults
    Tuned choice;
    if (ctx->forced) {
        choice.t = ctx->forced_t;
    } else if (flags & LVBH_AUTOTUNE) {
        auto it = ctx->tuned.find(tkey);
        if (it != ctx->tuned.end()) {
            choice = it->second;
        } else {
            // time every candidate (second of two runs, stage by stage) on this very batch
            cudaEvent_t e0 = ctx->ev[0], e1 = ctx->ev[LVBH_NUM_STAGES];
            float best = 0.f;
            for (uint32_t c = 0; c < 4; ++c) {
                const BatchPlan cp = plan(kCandidates[c]);
                float ms = 0.f;
                for (int rep = 0; rep < 2; ++rep) {
                    LVBH_CUDA(ctx, cudaEventRecord(e0, s));
                    LVBH_CUDA(ctx, enqueue_batch(ctx, tri, cp, seg_bounds != nullptr, out, s, false));
                    LVBH_CUDA(ctx, cudaEventRecord(e1, s));
                    LVBH_CUDA(ctx, cudaEventSynchronize(e1));
                    LVBH_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
                }
                choice.ms[c] = ms;
                if (c == 0 || ms < best) { best = ms; choice.t = kCandidates[c]; }
            }
            choice.candidates = 4;
            ctx->tuned[tkey] = choice;
            if (profile) cudaEventRecord(ctx->ev[0], s);
        }
    }
    ctx->last_tuned = choice;
    const BatchPlan bp = plan(choice.t);
    if (profile || (flags & LVBH_NO_GRAPH)) {
        const cudaError_t qe = enqueue_batch(ctx, tri, bp, seg_bounds != nullptr, out, s, profile);
        cudaError_t e = cudaGetLastError();
        if (qe != cudaSuccess) return cuda_fail(ctx, qe, "tree pass tensor map");
        if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel launch");
    } else {
        if (int rc = launch_batch_graph(ctx, tri, bp, seg_bounds != nullptr, out, s)) return rc;
    }
    ctx->ev_valid = profile;
    LVBH_CUDA(ctx, cudaMemcpyAsync(ctx->host_ctl, ctx->ctl, offsetof(Control, pad1),
                                   cudaMemcpyDeviceToHost, s));
    if (bounds_out)
        LVBH_CUDA(ctx, cudaMemcpyAsync(ctx->bh_ord, ctx->b_ord, num_segs * 6ull * 4,
                                       cudaMemcpyDeviceToHost, s));
    ctx->last_stream = s;
    ctx->last_out = out;
    ctx->last_hb = HostBounds{};
    ctx->last_hb.use = seg_bounds != nullptr;
    ctx->last_batch = true;
    ctx->last_segs = num_segs;
    ctx->last_bounds_out = bounds_out;
    ctx->pending = true;
    if (flags & LVBH_ASYNC) return LVBH_OK;
    return lvbh_sync(ctx);
}

int lvbh_set_tunables(lvbh_ctx *ctx, const lvbh_tunables *t) {
    if (!ctx) return LVBH_EINVAL;
    if (!t) {
        ctx->forced = false;
        return LVBH_OK;
    }
    if ((t->digit_bits != 8 && t->digit_bits != 10) || (t->tree_block != 128 && t->tree_block != 256) ||
        t->tree_ctas_per_sm > 8)
        return fail(ctx, LVBH_EINVAL, "tunables: digit_bits 8 or 10, tree_block 128 or 256, tree_ctas_per_sm <= 8");
    ctx->forced = true;
    ctx->forced_t = Tunables{(int)t->digit_bits, t->tree_block == 128 ? 7 : 8, (int)t->tree_ctas_per_sm};
    return LVBH_OK;
}

int lvbh_get_tunables(lvbh_ctx *ctx, lvbh_tunables *t, float *candidate_ms, uint32_t *num_candidates) {
    if (!ctx || !t) return LVBH_EINVAL;
    const Tuned &c = ctx->last_tuned;
    t->digit_bits = (uint32_t)c.t.digit_bits;
    t->tree_block = 1u << c.t.log_block;
    t->tree_ctas_per_sm = (uint32_t)c.t.tree_ctas;
    t->reserved = 0;
    if (num_candidates) *num_candidates = c.candidates;
    for (uint32_t i = 0; candidate_ms && i < c.candidates; ++i) candidate_ms[i] = c.ms[i];
    return LVBH_OK;
}

int lvbh_sync(lvbh_ctx *ctx) {
    if (!ctx) return LVBH_EINVAL;
    if (!ctx->pending) return LVBH_OK;
    DeviceGuard g(ctx->device);
    ctx->pending = false;
    cudaError_t e = cudaStreamSynchronize(ctx->last_stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
    const uint32_t err = ctx->host_ctl[offsetof(Control, aux_err) / 4] | ctx->host_ctl[offsetof(Control, err) / 4];
    if (ctx->last_batch) {
        if (ctx->last_bounds_out) {
            for (uint64_t i = 0; i < ctx->last_segs * 6ull; ++i) {
                const uint64_t sg = i / 6;
                if (ctx->last_hb.use && !std::isnan(ctx->bh_bounds[6 * sg])) {
                    ctx->last_bounds_out[i] = ctx->bh_bounds[i];
                } else {
                    const uint32_t o = ctx->bh_ord[i];
                    const bool empty = ctx->bh_rows[sg + 1].tri == ctx->bh_rows[sg].tri;
                    ctx->last_bounds_out[i] = empty ? 0.0f : ord_word_to_float((i % 6) < 3 ? ~o : o);
                }
            }
        }
    } else if (ctx->last_out) {
        if (ctx->last_hb.use) {
            std::memcpy(ctx->last_out->bounds, ctx->last_hb.v, sizeof ctx->last_hb.v);
        } else {
            const uint32_t *b = ctx->host_ctl + offsetof(Control, bounds_ord) / 4;
            for (int a = 0; a < 3; ++a) {
                ctx->last_out->bounds[a] = ord_word_to_float(~b[a]);
                ctx->last_out->bounds[3 + a] = ord_word_to_float(b[3 + a]);
            }
        }
    }
    if (err & ERR_BAD_INDEX) return fail(ctx, LVBH_EINVAL, "vertex index out of range");
    if (err & ERR_NONFINITE) return fail(ctx, LVBH_EINVAL, "non-finite vertex coordinate in the input");
    if (err & ERR_LOOKBACK_TIMEOUT) return fail(ctx, LVBH_ETIMEOUT, "radix sort look-back wait exceeded its bound");
    if (err & ERR_COPY_TIMEOUT) return fail(ctx, LVBH_ETIMEOUT, "leaf gather copy wait exceeded its bound");
    if (err & ERR_CLIMB) return fail(ctx, LVBH_EDEVICE, "refit climb exceeded the maximum tree depth");
    if (err & ERR_SORT_RANGE)
        return fail(ctx, LVBH_EDEVICE, "radix sort scatter target out of range (digit counts inconsistent with the keys)");
    return LVBH_OK;
}

int lvbh_test_stall_lookback(lvbh_ctx *ctx, uint32_t stall_tile, uint32_t spin_cycles) {
    if (!ctx) return LVBH_EINVAL;
    DeviceGuard g(ctx->device);
    if (int rc = finish_pending(ctx)) return rc;
    ctx->test_stall1 = stall_tile + 1u;  // UINT32_MAX -> 0: no tile stalls
    ctx->test_spin = spin_cycles;
    if (ctx->ctl) {
        const uint32_t test_words[2] = {ctx->test_stall1, ctx->test_spin};
        LVBH_CUDA(ctx, cudaMemcpy(ctx->ctl, test_words, sizeof test_words, cudaMemcpyHostToDevice));
    }
    return LVBH_OK;
}

int lvbh_release(lvbh_ctx *ctx, lvbh_result *res) {
    if (!res) return LVBH_EINVAL;
    if (!res->owned) return LVBH_OK;
    DeviceGuard g(ctx ? ctx->device : 0);
    if (ctx && ctx->pending && ctx->last_out == res) lvbh_sync(ctx);
    cudaFree(res->nodes);
    cudaFree(res->tris);
    cudaFree(res->parents);
    cudaFree(res->leaf_index);
    cudaFree(res->morton);
    res->nodes = res->tris = nullptr;
    res->parents = nullptr;
    res->leaf_index = res->morton = nullptr;
    res->owned = 0;
    return LVBH_OK;
}

int lvbh_stage_times(lvbh_ctx *ctx, float *ms_out) {
    if (!ctx || !ms_out) return LVBH_EINVAL;
    for (int i = 0; i < LVBH_NUM_STAGES; ++i) ms_out[i] = 0.0f;
    if (!ctx->ev_valid) return fail(ctx, LVBH_EINVAL, "no profiled build to report");
    DeviceGuard g(ctx->device);
    for (int i = 0; i < LVBH_NUM_STAGES; ++i) {
        float ms = 0.0f;
        cudaError_t e = cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]);
        if (e != cudaSuccess) { cudaGetLastError(); ms = 0.0f; }
        ms_out[i] = ms;
    }
    return LVBH_OK;
}

int lvbh_copy_to_host(lvbh_ctx *ctx, void *dst_host, const void *src_device, size_t bytes,
                      void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (bytes && (!dst_host || !src_device)) return fail(ctx, LVBH_EINVAL, "NULL copy pointer");
    if (!bytes) return LVBH_OK;
    DeviceGuard g(ctx->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    LVBH_CUDA(ctx, cudaMemcpyAsync(dst_host, src_device, bytes, cudaMemcpyDeviceToHost, s));
    LVBH_CUDA(ctx, cudaStreamSynchronize(s));
    return LVBH_OK;
}

size_t lvbh_scratch_bytes(uint32_t num_tris) {
    return arena_bytes(num_tris < 4096 ? 4096 : num_tris);
}

const char *lvbh_last_error(const lvbh_ctx *ctx) {
    if (!ctx) return "no context";
    return ctx->err.c_str();
}

int lvbh_trace(lvbh_ctx *ctx, const void *nodes, const void *tris, uint32_t num_tris,
               const float *rays, uint32_t num_rays, int32_t *hit_prim, float *hit_t,
               uint32_t *max_stack, void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (num_rays && (!rays || !hit_prim || !hit_t)) return fail(ctx, LVBH_EINVAL, "NULL ray buffer");
    if (num_tris && (!nodes || !tris)) return fail(ctx, LVBH_EINVAL, "NULL tree buffer");
    DeviceGuard g(ctx->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!ctx->trace_counter) LVBH_CUDA(ctx, cudaMalloc(&ctx->trace_counter, sizeof(uint32_t)));
    launch_trace(static_cast<const float4 *>(nodes), static_cast<const float4 *>(tris), num_tris,
                 reinterpret_cast<const float4 *>(rays), num_rays, hit_prim, hit_t, max_stack,
                 ctx->trace_counter, s);
    LVBH_CUDA(ctx, cudaGetLastError());
    LVBH_CUDA(ctx, cudaStreamSynchronize(s));
    return LVBH_OK;
}

int lvbh_pt_sample(lvbh_ctx *ctx, const void *nodes, const void *tris, uint32_t num_tris,
                   const float *state_in, float *state_out, uint32_t width, uint32_t height,
                   const lvbh_pt_frame *frame, void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (!frame) return fail(ctx, LVBH_EINVAL, "frame is NULL");
    const uint64_t pixels = (uint64_t)width * height;
    if (pixels >= (1ull << 31)) return fail(ctx, LVBH_EINVAL, "image too large");
    if (pixels && (!state_out || (frame->rst == 0.0f && !state_in))) return fail(ctx, LVBH_EINVAL, "NULL state buffer");
    if (num_tris && (!nodes || !tris)) return fail(ctx, LVBH_EINVAL, "NULL tree buffer");
    if (num_tris > LVBH_MAX_TRIS) return fail(ctx, LVBH_EINVAL, "num_tris exceeds LVBH_MAX_TRIS");
    if (!pixels) return LVBH_OK;
    DeviceGuard g(ctx->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!ctx->trace_counter) LVBH_CUDA(ctx, cudaMalloc(&ctx->trace_counter, sizeof(uint32_t)));
    PtFrame f{};
    for (int a = 0; a < 3; ++a) { f.pos[a] = frame->pos[a]; f.lat[a] = frame->lat[a]; }
    f.rst = frame->rst;
    f.width = width;
    f.height = height;
    f.sw_x = (float)width;
    f.sw_y = (float)height;
    // the constants the shader bakes in (pathtracer.js:477-485, :716): aspect = w / h,
    // sinfov = sin(.5 * fov * Pi / 180.f) with the argument in float, pow(.3f, 2.2)
    f.aspect = (float)((double)width / (double)height);
    const float half_fov = ((0.5f * 60.0f) * (float)3.14159265358979323846) / 180.0f;
    f.sinfov = (float)std::sin((double)half_fov);
    f.powc = (float)std::pow((double)0.3f, (double)2.2f);
    launch_pt_step(static_cast<const float4 *>(nodes), static_cast<const float4 *>(tris), num_tris,
                   reinterpret_cast<const float4 *>(state_in), reinterpret_cast<float4 *>(state_out), f,
                   ctx->trace_counter, s);
    LVBH_CUDA(ctx, cudaGetLastError());
    LVBH_CUDA(ctx, cudaStreamSynchronize(s));
    return LVBH_OK;
}

int lvbh_parse_obj(lvbh_ctx *ctx, const char *text, uint64_t bytes, uint32_t flags,
                   const float **tri_out, uint32_t *num_tris, double *bounds6, uint64_t *err_line,
                   void *stream) {
    if (!ctx) return LVBH_EINVAL;
    if (!tri_out || !num_tris || !bounds6 || !err_line) return fail(ctx, LVBH_EINVAL, "NULL output pointer");
    *err_line = 0;
    if (bytes && !text) return fail(ctx, LVBH_EINVAL, "text is NULL");
    if (bytes > LVBH_OBJ_MAX_BYTES) return fail(ctx, LVBH_EINVAL, "text exceeds LVBH_OBJ_MAX_BYTES");
    DeviceGuard g(ctx->device);
    if (ctx->pending) LVBH_CUDA(ctx, cudaStreamSynchronize(ctx->last_stream));
    return obj_parse(ctx->obj, text, bytes, (flags & LVBH_INPUT_HOST) != 0, tri_out, num_tris, bounds6,
                     err_line, static_cast<cudaStream_t>(stream), ctx->err);
}

}  // extern "C"
