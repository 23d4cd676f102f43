// lvbh_internal.h - launch wrappers shared between the kernel files and the C-ABI layer.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

struct lvbh_ctx;

namespace lvbh {

// Radix sort geometry of the build: Morton keys are below 2^30 (split_3's last mask tops out
// at bit 27, shifted left by 2), so three passes of 10-bit digits cover every key bit.
constexpr int kDigitBits = 10;
constexpr int kDigits = 1 << kDigitBits;
constexpr int kSortPasses = 3;
// Full 32-bit keys (the allocation-free sort of caller keys): four passes of 8-bit digits.
constexpr int kDigitBits32 = 8;
constexpr int kDigits32 = 1 << kDigitBits32;
constexpr int kSortPasses32 = 4;
constexpr int kHistWords = kSortPasses * kDigits;  // also holds the 4 x 256 counts of 32-bit keys
static_assert(kSortPasses32 * kDigits32 <= kHistWords, "histogram space");
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;                       // keys per thread
constexpr int kSortTile = kSortThreads * kSortItems; // keys per tile (4096)

__host__ __device__ inline uint32_t sort_tiles(uint32_t n) { return (n + kSortTile - 1) / kSortTile; }

// The plain build's sort scratch: per tile of kSortTile keys its kDigits counts of the pass's
// digit, per chunk of sort_chunk_tiles(n) tiles their sum, per chunk the output offsets.  A
// chunk is one block of the per-chunk kernels (Morton keys, tile histograms): 8 tiles when that
// still gives kChunkFill blocks (two per SM), fewer for smaller sorts.
constexpr int kSortChunkTiles = 8;
constexpr uint32_t kChunkFill = 296;
__host__ __device__ inline uint32_t sort_chunk_tiles(uint32_t n) {
    const uint32_t t = sort_tiles(n);
    return t >= 8 * kChunkFill ? 8u : t >= 4 * kChunkFill ? 4u : t >= 2 * kChunkFill ? 2u : 1u;
}
__host__ __device__ inline uint32_t sort_chunks(uint32_t n) {
    const uint32_t ct = sort_chunk_tiles(n);
    return (sort_tiles(n) + ct - 1) / ct;
}
// An upper bound of sort_chunks(m) over every m <= n (scratch sized for n serves them all).
inline uint32_t sort_chunks_bound(uint32_t n) {
    const uint32_t t = sort_tiles(n), c8 = (t + 7) / 8, lo = 2 * kChunkFill;
    const uint32_t b = c8 > lo ? c8 : lo;
    return b < t ? b : t;
}
inline uint32_t *sort_chunk_sums(uint32_t *scratch, uint32_t n) {
    return scratch + (size_t)sort_tiles(n) * kDigits;
}

// Tree/refit pass: leaves per block of the in-block tree pass (one thread each); open nodes a
// block can leave to the straddling pass (at most 2 x the tree depth 64).
constexpr int kLogEmitBlock = 8;  // the plain build's tree blocks (a batched build may use 7)
constexpr int kEmitBlock = 1 << kLogEmitBlock;
constexpr int kOpenCap = 128;

// A complete subtree handed from one level of the tree pass to the next: box min + link,
// box max + the separator d after it (d[xr]), its leaf range and the separator before it
// (d[xl - 1]).
struct __align__(16) OpenItem {
    float4 lo;
    float4 hi;
    int xl, xr, pad0, pad1;  // pad0: d[xl - 1]
};

constexpr int kHistParts = 16;

// Per-build control block in device memory.  Everything from `err` on is zeroed by one memset
// at the start of a build; `aux_err` collects errors of steps that run before that memset (the
// indexed-mesh gather) and is cleared by the host before them.  The two test words at the front
// (lvbh_test_stall_lookback) persist across builds: when test_stall_tile1 is not zero, sort
// tile test_stall_tile1 - 1 of every look-back pass publishes nothing, so the tiles after it
// wait until their bound runs out; test_spin_limit, when not zero, replaces kSpinLimitCycles
// as that bound.  Both are zero in normal use.
struct Control {
    uint32_t test_stall_tile1;
    uint32_t test_spin_limit;
    uint32_t aux_err;
    uint32_t err;
    uint32_t tile_counter[kSortPasses32];
    uint32_t pad0[2];
    uint32_t bounds_ord[6];   // scene min (ord_hi) and max (ord_lo), see lvbh_device.cuh
    uint32_t pad1[2];
    uint32_t hist[kHistWords];  // global digit counts of the unsorted keys, pass-major
    // The plain build's global digit counts in kHistParts partial rows per pass: each per-chunk
    // block adds its chunk's counts into row (chunk % kHistParts), so that hundreds of blocks
    // finishing together do not queue on one address per digit; the chunk scan sums the rows.
    uint32_t hist_part[kSortPasses][kHistParts][kDigits];
};

struct HostBounds {
    float v[6];
    int use;  // 1 = quantise with v; 0 = with the device reduction in Control::bounds_ord
};

// Batched builds: segments (meshes) laid end to end in one soup.  Row s of the segment table
// holds segment s's first triangle, first sort tile and first tree block; row num_segs holds
// the totals.  Sort tiles (kSortTile keys) and tree blocks (kEmitBlock leaves) never cross a
// segment boundary, so each tile or block works on one segment with segment-local indices.
struct __align__(16) SegRow {
    uint32_t tri, tile, blk, grp;  // first triangle, sort tile, tree block, straddling group
};

struct BatchPlan {
    const SegRow *rows;        // num_segs + 1 rows (device)
    const uint32_t *tile_seg;  // segment of each sort tile (device, `tiles` entries)
    const uint32_t *blk_seg;   // segment of each tree block (device, `blocks` entries)
    const uint32_t *grp_seg;   // segment of each straddling-pass group (device, `groups` entries)
    uint32_t num_segs, tiles, blocks, total, groups;
    int digit_bits;            // sort digit width: 10 (three passes) or 8 (four passes)
    int log_block;             // tree blocks of 2^log_block leaves: 8 or 7
    int tree_ctas_per_sm;      // persistent tree grid: CTAs per SM (0 = the most that fit)
};

int sm_count();

// Launches a kernel that begins with chain_wait().  Chained (programmatic stream
// serialisation), its launch overlaps the completion of the kernel before it on the stream,
// which saves most of the launch gap at each kernel boundary of a build; otherwise it launches
// in plain stream order.
template <typename... P, typename... A>
cudaError_t launch_chained(bool chain, void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                           cudaStream_t s, A &&...args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = chain ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<A &&>(args)...);
}

// Whether a one-mesh build of n triangles chains its kernels.  Measured on B200: 4,096 meshes of
// 64 to 262,144 triangles built one launch sequence each took 373 ms chained against 451 ms;
// graph-replayed builds of clustered triangles took the same time either way up to 2^18 and at
// 2^21 to 2^23, less chained at 2^20 (0.237 -> 0.232 ms) and a little more at 2^24 (1.7035 ->
// 1.7066 ms, within the run-to-run spread), so the 16.7 M build keeps plain stream order.
constexpr uint32_t kChainMaxTris = 1u << 22;
inline bool chain_build(uint32_t n) { return n <= kChainMaxTris; }

// Server support (api.cu): size a context's scratch for batched builds of up to max_tris
// triangles in up to max_segs meshes, and report the device bytes the context holds.
int ctx_reserve_batch(lvbh_ctx *ctx, uint32_t max_tris, uint32_t max_segs);
size_t ctx_device_bytes(const lvbh_ctx *ctx);

// K1a: scene box over every vertex of the 48-byte triangle soup.
void launch_bounds(const float4 *tri, uint32_t n, Control *ctl, cudaStream_t s);
// K1b: triangle box centroid -> Morton key (input order), the first sort pass's tile
// histograms, chunk sums (sort_scratch) and global digit counts (ctl->hist_part, zero before); flags
// non-finite vertices in ctl->err and advances the build epoch *epoch used by K3c.
void launch_morton(const float4 *tri, uint32_t n, HostBounds hb, Control *ctl,
                   uint32_t *keys_out, uint32_t *epoch, uint32_t *sort_scratch, cudaStream_t s);
// K1b over the sort-tile chunks [c0, c1) only (chunk = sort_chunk_tiles(n) tiles): the keys of
// a soup uploaded chunk by chunk, each part launched once its triangles have landed.
void launch_morton_chunks(const float4 *tri, uint32_t n, HostBounds hb, Control *ctl, uint32_t *keys,
                          uint32_t *epoch, uint32_t *sort_scratch, uint32_t c0, uint32_t c1, cudaStream_t s);
// K1a + K1b split for a soup whose box is reduced on the device: K1a over triangles [t0, t1)
// also stores each triangle's centroid (cen[t], cen[stride + t], cen[2 stride + t]); K1b then
// quantises the centroids (12 bytes per triangle instead of the 48-byte soup).
void launch_bounds_cen(const float4 *tri, uint32_t t0, uint32_t t1, float *cen, uint32_t cen_stride,
                       Control *ctl, cudaStream_t s);
void launch_morton_cen(const float *cen, uint32_t cen_stride, uint32_t n, Control *ctl, uint32_t *keys,
                       uint32_t *epoch, uint32_t *sort_scratch, cudaStream_t s);
cudaError_t morton_init();  // once per device, before the first launch
// K2: one reduce-then-scan pass over 10-bit digit `pass` (0..2) of 30-bit keys.  counted: the
// tile histograms, chunk sums and global digit counts (ctl->hist_part) of this pass are there
// already (K1b makes those of pass 0); otherwise the pass's tile-histogram kernel makes them
// (ctl->hist_part of the pass zero before).  vals_in == nullptr generates the
// identity.  scratch: sort_scratch_words(n) words, no initialisation needed.
size_t sort_scratch_words(uint32_t n);
void launch_sort_pass(const uint32_t *keys_in, const uint32_t *vals_in, uint32_t *keys_out,
                      uint32_t *vals_out, uint32_t n, int pass, bool counted, Control *ctl,
                      uint32_t *scratch, cudaStream_t s);
// The same over 8-bit digit `pass` (0..3) of full 32-bit keys (counts in ctl->hist pass-major,
// 256 per pass; look-back words kSortPasses32 * sort_tiles(n) * kDigits32).
void launch_onesweep32(const uint32_t *keys_in, const uint32_t *vals_in, uint32_t *keys_out,
                       uint32_t *vals_out, uint32_t n, int pass, Control *ctl, uint32_t *lookback,
                       cudaStream_t s);
cudaError_t sort_init();  // once per device, before the first launch
// K3: leaf gather + rearrange + in-block radix tree and refit (K3b), straddling nodes (K3c)
// -> BVH nodes, parent links, sorted triangles.  Scratch: items (emit_groups(n) * kOpenCap)
// and counts (emit_groups(n)), arrive (n words, zero or older epochs), pend (2n float4),
// pend_d (n bytes); *epoch is this build's epoch (advanced by K1b).
size_t emit_groups(uint32_t n, int log_eb = kLogEmitBlock);
// Groups of the straddling pass's first level over `blocks` tree blocks of one segment.
inline uint32_t straddle_groups(uint32_t blocks) { return (blocks + 15u) / 16u; }
cudaError_t emit_init();  // once per device, before the first launch
// ev (may be nullptr): three events, recorded before K3b, after K3b and after K3c.  An error:
// the soup's tensor map (K3b's gather) could not be made; nothing was launched.
cudaError_t launch_emit(const float4 *tri, const uint32_t *perm, const uint32_t *keys, uint32_t n,
                        float4 *otri, float4 *nodes, int32_t *parents, OpenItem *items,
                        uint32_t *counts, uint32_t *arrive, float4 *pend, uint8_t *pend_d,
                        const uint32_t *epoch, Control *ctl, cudaStream_t s, cudaEvent_t *ev);
// Batched forms of K1a, K1b, K2 and K3 over the segments of `bp`.  seg_ord holds 6 ordered
// bound words per segment (zeroed before K1a; min at 0-2 as ~ord_lo, max at 3-5 as ord_lo),
// seg_hist 4 x 256 digit counts per segment (zeroed before K1b); host_bounds, when not null,
// holds 6 floats per segment that replace the device reduction for every segment whose first
// value is not NaN.  K2's look-back words: bp.tiles * 256 per pass, zeroed before the build.
void launch_seg_tables(const SegRow *rows, uint32_t num_segs, uint32_t *tile_seg,
                       uint32_t *blk_seg, uint32_t *grp_seg, cudaStream_t s);
void launch_bounds_batch(const BatchPlan &bp, const float4 *tri, const float *host_bounds,
                         uint32_t *seg_ord, cudaStream_t s);
// seg_hist: kHistWords per segment, pass-major (bp.digit_bits wide digits).
void launch_morton_batch(const BatchPlan &bp, const float4 *tri, const float *host_bounds,
                         const uint32_t *seg_ord, uint32_t *seg_hist, Control *ctl,
                         uint32_t *keys_out, uint32_t *epoch, cudaStream_t s);
void launch_onesweep_batch(const BatchPlan &bp, const uint32_t *keys_in, const uint32_t *vals_in,
                           uint32_t *keys_out, uint32_t *vals_out, int pass,
                           const uint32_t *seg_hist, Control *ctl, uint32_t *lookback,
                           cudaStream_t s);
// items / counts: bp.blocks * kOpenCap / bp.blocks entries (open items per tree block).
// Errors as launch_emit.
cudaError_t launch_emit_batch(const BatchPlan &bp, const float4 *tri, const uint32_t *perm,
                              const uint32_t *keys, float4 *otri, float4 *nodes, int32_t *parents,
                              OpenItem *items, uint32_t *counts, uint32_t *arrive, float4 *pend,
                              uint8_t *pend_d, const uint32_t *epoch, Control *ctl, cudaStream_t s,
                              cudaEvent_t *ev);
// Indexed mesh -> 48-byte soup (pad 0).  An index >= num_verts sets ERR_BAD_INDEX in
// *err and gathers zeros instead of reading out of bounds.
void launch_gather_indexed(const float *xyz, uint32_t num_verts, const uint32_t *idx3,
                           uint32_t n, float4 *tri, uint32_t *err, cudaStream_t s);
// K5: closest-hit traversal (persistent, rays fetched from *counter, which it zeroes first).
void launch_trace(const float4 *nodes, const float4 *tris, uint32_t n, const float4 *rays,
                  uint32_t num_rays, int32_t *hit_prim, float *hit_t, uint32_t *max_stack,
                  uint32_t *counter, cudaStream_t s);

// The indexed leaf format (a mesh of 16-byte vertex rows + index triples): K1a over the
// vertices the triangles use, K1b gathering each triangle's rows, the sorted index triples
// (sidx[i] = idx3[perm[i]]), and K3 reading leaves through sidx.
void launch_bounds_mesh(const float4 *verts, uint32_t nverts, const uint32_t *idx3, uint32_t n, Control *ctl,
                        cudaStream_t s);
void launch_morton_mesh(const float4 *verts, uint32_t nverts, const uint32_t *idx3, uint32_t n, HostBounds hb,
                        Control *ctl, uint32_t *keys, uint32_t *epoch, uint32_t *sort_scratch, cudaStream_t s);
void launch_leaf_idx(const uint32_t *idx3, const uint32_t *perm, uint32_t n, uint32_t *sidx, cudaStream_t s);
void launch_emit_mesh(const float4 *verts, uint32_t num_verts, const uint32_t *sidx, const uint32_t *keys,
                      uint32_t n, float4 *nodes, int32_t *parents, OpenItem *items, uint32_t *counts,
                      uint32_t *arrive, float4 *pend, uint8_t *pend_d, const uint32_t *epoch, Control *ctl,
                      cudaStream_t s, cudaEvent_t *ev);
// K5 over the indexed leaf format: leaf i's vertices are verts[sidx[3i..3i+2]].
void launch_trace_mesh(const float4 *nodes, const float4 *verts, uint32_t num_verts, const uint32_t *sidx, uint32_t n,
                       const float4 *rays, uint32_t num_rays, int32_t *hit_prim, float *hit_t,
                       uint32_t *max_stack, uint32_t *counter, cudaStream_t s);

// Path-trace bounce (trace.cu): the uniform buffer (pos, rst, lat) and the constants the
// reference's shader bakes in (image size, aspect, sin(fov / 2), pow(.3, 2.2)).
struct PtFrame {
    float pos[3], rst, lat[3];
    uint32_t width, height;
    float sw_x, sw_y, aspect, sinfov, powc;
};
// One bounce of every pixel: state planes o, d, t, b of width x height float4 each.
void launch_pt_step(const float4 *nodes, const float4 *tris, uint32_t n, const float4 *state_in,
                    float4 *state_out, const PtFrame &f, uint32_t *counter, cudaStream_t s);

// OBJ ingest (obj.cu): device memory of one parse, grown on demand and held by the context.
struct ObjScratch {
    void *text = nullptr;  // staged host text, newline counts, control block
    size_t text_bytes = 0;
    void *lines = nullptr;  // per-line arrays
    size_t lines_bytes = 0;
    void *soup = nullptr;  // model-0 vertices (double) and the triangle soup
    size_t soup_bytes = 0;
    void *host = nullptr;  // pinned readback
};
// OBJ text -> triangle soup + bounds (lvbh_parse_obj).  *err_line: the 1-based line whose
// statement the parser rejects, 0 for a failure found after parsing (LVBH_EINVAL for both).
int obj_parse(ObjScratch &sc, const char *text, uint64_t bytes, bool host_text,
              const float **tri_out, uint32_t *num_tris, double *bounds6, uint64_t *err_line,
              cudaStream_t s, std::string &err);
void obj_free(ObjScratch &sc);

}  // namespace lvbh
