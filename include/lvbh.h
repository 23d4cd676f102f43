/*
 * lvbh.h - C ABI of the B200 (sm_100a) LBVH builder.
 *
 * This library is a drop-in for the BVH build path of AddisonPrairie/WebGPU-LVBH-demo:
 *
 *   initBVHBuild(device) -> { build }                        scripts/bvh/build-bvh.js:1-10
 *   async build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS)
 *       -> { BVH_BUFFER, O_TRIANGLE_BUFFER }                 scripts/bvh/build-bvh.js:12-66
 *
 * Every entry point takes plain pointers and sizes; no C++ or framework type crosses
 * the boundary, and no exception escapes it.  Status codes replace the reference's
 * `console.warn(...); return undefined` (scripts/bvh/kernels/aabb-z-idx.js:58-61,
 * radix-tree.js:51-54, rearrange.js:58-66).
 *
 * Layouts (identical to what scripts/pathtracer/pathtracer.js:441-459 traverses):
 *
 *   Triangle (input and output), 48 B:  float v0[3], pad, v1[3], pad, v2[3], pad
 *        (WGSL vec3f members at 16-byte alignment, scripts/bvh/kernels/aabb-z-idx.js:153-157;
 *         pad words are ignored on input and copied unchanged into the output).
 *
 *   BVHNode, 64 B (scripts/bvh/kernels/bvh-up-pass.js:161-178):
 *        word  0- 2  left  box min      word  3  l_child
 *        word  4- 6  left  box max      word  7  f_1
 *        word  8-10  right box min      word 11  r_child
 *        word 12-14  right box max      word 15  f_2
 *     A child >= 0 is an internal node index; a child < 0 is the leaf -(sorted_pos + 1),
 *     i.e. triangle `sorted_pos` of the output triangle buffer.  Node 0 is the root.  The
 *     buffer holds N records and record N-1 is all zero, as in the reference.
 *     Canonical form: the left slot holds the Karras left child (the lower key range),
 *     f_1 = 2 and f_2 = 0 for every internal node (f_1 = 1 for the single node of an N = 1
 *     build).  The reference fills the slots in arrival order and leaves an arrival/spin
 *     count in f_1; a tree of it equals this one after sorting each node's two slots by
 *     child range and masking words 7 and 15.
 *
 *   parents, int32 x 2N (scripts/bvh/kernels/radix-tree.js:57-60,146-156):
 *        [0, N-2]  parent of internal node i      [N, 2N-1]  parent of leaf (sorted pos) i-N
 *        slots 0 and N-1 hold 0.
 *   leaf_index, uint32 x N: sorted position -> input triangle index (the reference's IDX_BUFFER).
 *   morton, uint32 x N: the sorted Morton keys (the reference's Z_IDX_BUFFER after the sort).
 *
 * Memory: all result buffers are device memory of the context's device.  Input may be host
 * or device memory (LVBH_INPUT_HOST).
 */
#ifndef LVBH_H
#define LVBH_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LVBH_API __attribute__((visibility("default")))
#else
#define LVBH_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define LVBH_OK        0
#define LVBH_EINVAL    1  /* bad argument: NULL pointer, size out of range, non-finite vertex */
#define LVBH_ENOMEM    2  /* device or pinned allocation failed, or the memory budget is exceeded */
#define LVBH_ETIMEOUT  3  /* a device-side wait gave up after its bound (error word set by a kernel) */
#define LVBH_ECUDA     4  /* a CUDA runtime call failed; lvbh_last_error() has the text */
#define LVBH_EBUSY     5  /* serving: queue full / request not finished yet */
#define LVBH_EDEVICE   6  /* a kernel reported an inconsistent structure (bounded climb exceeded) */
#define LVBH_ERANGE    7  /* a size beyond a fixed capacity (lvbh_sort_pairs_noalloc) */
#define LVBH_EPARSE    8  /* lvbh_parse_obj: the text is one the reference's OBJ parser throws on */

/* ---- build flags ------------------------------------------------------------------- */
#define LVBH_INPUT_HOST    0x1u  /* input pointers are host memory: copied to the device inside the call */
#define LVBH_ASYNC         0x2u  /* return after enqueueing; call lvbh_sync() before reading results/status */
#define LVBH_OUT_CALLER    0x4u  /* result pointers in *out are caller-owned device buffers to fill */
#define LVBH_PROFILE       0x8u  /* record per-stage CUDA events; read them with lvbh_stage_times() */
#define LVBH_NO_GRAPH      0x10u /* launch stage by stage instead of replaying a cached CUDA graph */
#define LVBH_AUTOTUNE      0x20u /* lvbh_build_batched: pick the tunables by timing the candidates
                                    on the first batch of each mesh-size histogram (cached) */

/* Largest triangle count one build accepts (2^29: keeps every index sum of the tree search
 * inside int32 and the look-back counts inside their 30-bit field; a build this size needs
 * about 100 GB of device memory). */
#define LVBH_MAX_TRIS  ((uint32_t)1 << 29)

/* Stage indices for lvbh_stage_times(). */
#define LVBH_STAGE_UPLOAD  0  /* host->device copy of the input (LVBH_INPUT_HOST only) */
#define LVBH_STAGE_BOUNDS  1  /* scene box reduction with the triangle centroids (skipped when bounds are supplied) */
#define LVBH_STAGE_MORTON  2  /* triangle centroid -> 30-bit Morton key + digit histograms */
#define LVBH_STAGE_SORT    3  /* stable LSD radix sort of (key, triangle index) */
#define LVBH_STAGE_GATHER  4  /* empty: the leaf gather runs inside the tree stage */
#define LVBH_STAGE_TREE    5  /* leaf gather + rearrange, radix tree + box refit inside each block */
#define LVBH_STAGE_TOP     6  /* radix tree + box refit of the nodes that straddle blocks */
#define LVBH_NUM_STAGES    7

typedef struct lvbh_ctx lvbh_ctx;

typedef struct lvbh_config {
    int      device;        /* CUDA device ordinal; -1 = the calling thread's current device */
    uint32_t reserve_tris;  /* pre-size the scratch arena for this many triangles (0 = on demand) */
    uint64_t reserved[4];   /* must be zero */
} lvbh_config;

typedef struct lvbh_result {
    uint32_t  num_tris;     /* N */
    uint32_t  num_nodes;    /* N: BVHNode records in `nodes` (record N-1 is zero) */
    void     *nodes;        /* BVH_BUFFER: 64 B x N */
    void     *tris;         /* O_TRIANGLE_BUFFER: 48 B x N, sorted order */
    int32_t  *parents;      /* 2N */
    uint32_t *leaf_index;   /* N */
    uint32_t *morton;       /* N */
    float     bounds[6];    /* scene min xyz, max xyz used for quantisation (filled at sync) */
    uint32_t  owned;        /* 1 when the library allocated the buffers (free with lvbh_release) */
} lvbh_result;

/* Replaces initBVHBuild(device) (scripts/bvh/build-bvh.js:1-10): binds a context to a device.
 * `cfg` may be NULL (current device, no reservation). */
LVBH_API int  lvbh_create(lvbh_ctx **ctx, const lvbh_config *cfg);
/* Frees the context and its scratch arena.  Results it allocated stay valid until released. */
LVBH_API void lvbh_destroy(lvbh_ctx *ctx);

/* Replaces build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS) (scripts/bvh/build-bvh.js:12-66).
 *   tri_array    12 floats per triangle (48 B stride), host memory when LVBH_INPUT_HOST is set.
 *   num_tris     N; 0 gives an empty result, as in the reference.
 *   model_bounds 6 host floats {min x,y,z, max x,y,z} used for quantisation exactly as the
 *                reference's uniform (aabb-z-idx.js:113-132); NULL = reduce min/max over all
 *                vertices on the device (what parse-obj.js:27-53 computes on the host).
 *   flags        LVBH_* build flags.
 *   out          receives the result.  Without LVBH_OUT_CALLER the library allocates the
 *                buffers (stream-ordered) and the caller frees them with lvbh_release().
 *   stream       cudaStream_t to run on (NULL = the legacy default stream).
 * Synchronous unless LVBH_ASYNC: the call returns once results are ready and device-side
 * checks (non-finite input, bounded waits) have been read back. */
LVBH_API int  lvbh_build_soup(lvbh_ctx *ctx, const float *tri_array, uint32_t num_tris,
                     const float *model_bounds, uint32_t flags, lvbh_result *out, void *stream);

/* Indexed-mesh form of lvbh_build_soup (vertex and index buffers in): vertices are packed
 * float3 (12 B), indices are uint32 triples.  The triangles are gathered on the
 * device into the same 48 B layout (pad words = 0), then built exactly as lvbh_build_soup. */
LVBH_API int  lvbh_build_indexed(lvbh_ctx *ctx, const float *xyz, uint32_t num_verts,
                        const uint32_t *idx3, uint32_t num_tris, const float *model_bounds,
                        uint32_t flags, lvbh_result *out, void *stream);

/* Indexed leaf format: the same tree from an indexed mesh without any 48-byte triangle copy.
 * No counterpart in the reference, whose rearrange pass (scripts/bvh/kernels/rearrange.js:
 * 162-169) copies every triangle into O_TRIANGLE_BUFFER; here a leaf refers to its vertices.
 *   verts4     num_verts rows of 16 B {x, y, z, pad} (16-byte aligned when device memory)
 *   idx3       num_tris uint32 triples into verts4
 * nodes, parents, leaf_index and morton equal those of lvbh_build_soup over the triangles the
 * mesh spells out (bounds: min / max over the vertices the triangles use).  out->tris receives,
 * per sorted leaf, the triangle's three vertex indices (12 B per triangle, i.e. idx3 of
 * leaf_index) instead of its 48-byte rows: leaf -(i+1) of a node has the vertices
 * verts4[tris[3i]], verts4[tris[3i+1]], verts4[tris[3i+2]].  With LVBH_OUT_CALLER, out->tris
 * must hold 12 N bytes (4-byte aligned).  An index >= num_verts fails the build with
 * LVBH_EINVAL. */
LVBH_API int  lvbh_build_mesh(lvbh_ctx *ctx, const float *verts4, uint32_t num_verts,
                        const uint32_t *idx3, uint32_t num_tris, const float *model_bounds,
                        uint32_t flags, lvbh_result *out, void *stream);

/* Batched build: num_segs independent meshes laid end to end in one triangle soup, built in
 * one stream-ordered launch sequence (replayed as a cached CUDA graph) instead of one
 * build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS) per mesh (scripts/bvh/build-bvh.js:12-66 called
 * num_segs times).
 *   tri_array    12 floats per triangle for all meshes (host memory with LVBH_INPUT_HOST).
 *   seg_offsets  HOST memory, num_segs + 1 entries: mesh s is triangles
 *                [seg_offsets[s], seg_offsets[s+1]); seg_offsets[0] = 0, non-decreasing,
 *                total = seg_offsets[num_segs] <= LVBH_MAX_TRIS.  Empty meshes are allowed.
 *   seg_bounds   HOST memory, 6 floats per mesh used as that mesh's MODEL_BOUNDS, or NULL =
 *                each mesh's own vertex box reduced on the device.  A mesh whose first value
 *                is NaN is reduced on the device too (bounds given for some meshes only).
 *   bounds_out   HOST memory, 6 floats per mesh receiving the bounds each mesh was quantised
 *                with (written when the build completes: at lvbh_sync with LVBH_ASYNC), or NULL.
 *   out          total-sized result.  Mesh s (n_s triangles from o_s = seg_offsets[s]) owns
 *                node records and sorted triangles [o_s, o_s + n_s), parents entries
 *                [2 o_s, 2 o_s + 2 n_s) and leaf_index / morton entries [o_s, o_s + n_s); every
 *                index inside them is local to the mesh, so each slice is bit-identical to
 *                lvbh_build_soup of that mesh alone and is a BVH_BUFFER / O_TRIANGLE_BUFFER of
 *                its own.  out->bounds is zeroed.
 * Flags, stream and synchronisation as for lvbh_build_soup. */
LVBH_API int  lvbh_build_batched(lvbh_ctx *ctx, const float *tri_array, const uint32_t *seg_offsets,
                        uint32_t num_segs, const float *seg_bounds, float *bounds_out,
                        uint32_t flags, lvbh_result *out, void *stream);

/* Tunables of batched builds (no counterpart in the reference, whose kernels hard-code
 * WG_SIZE = 64 and 2-bit digits).  With LVBH_AUTOTUNE, lvbh_build_batched keys the meshes'
 * size histogram (per power-of-two size class, the bit length of the number of meshes in it),
 * and on the first batch with a new key times each candidate - digit width {10, 8} x tree block
 * {256, 128} - on that batch itself, then builds every batch with that key with the fastest.
 * Without it the defaults are used (10-bit digits, 256-leaf blocks).  Every choice gives the
 * same result words. */
typedef struct lvbh_tunables {
    uint32_t digit_bits;        /* radix sort digit width: 10 (three passes) or 8 (four passes) */
    uint32_t tree_block;        /* sorted leaves per tree block: 256 or 128 */
    uint32_t tree_ctas_per_sm;  /* tree-pass CTAs per SM (persistent grid); 0 = as many as fit */
    uint32_t reserved;
} lvbh_tunables;
/* Forces the tunables of later batched builds on this context; NULL returns to LVBH_AUTOTUNE /
 * defaults. */
LVBH_API int  lvbh_set_tunables(lvbh_ctx *ctx, const lvbh_tunables *t);
/* The tunables of the context's last batched build and, when that build tuned, the times of
 * the candidates (ms, up to 4, in the order listed above; *num_candidates = 0 otherwise). */
LVBH_API int  lvbh_get_tunables(lvbh_ctx *ctx, lvbh_tunables *t, float *candidate_ms,
                                uint32_t *num_candidates);

/* Waits for the context's last build and returns its device-side status (LVBH_OK,
 * LVBH_EINVAL for non-finite vertices, LVBH_ETIMEOUT, LVBH_EDEVICE).  Fills out->bounds
 * of the result passed to that build when it is still reachable.  Every build entry point
 * first finishes the context's pending LVBH_ASYNC build this way; when that build failed, the
 * entry point returns its status (lvbh_last_error says so) and starts no new build. */
LVBH_API int  lvbh_sync(lvbh_ctx *ctx);

/* Frees library-allocated result buffers (no-op for LVBH_OUT_CALLER results). */
LVBH_API int  lvbh_release(lvbh_ctx *ctx, lvbh_result *res);

/* Per-stage device times (ms) of the last build made with LVBH_PROFILE, LVBH_NUM_STAGES
 * entries, after lvbh_sync(). */
LVBH_API int  lvbh_stage_times(lvbh_ctx *ctx, float *ms_out);

/* Copies `bytes` from device memory of the context's device to host memory and waits (for FFI
 * callers that do not link the CUDA runtime themselves).  stream: cudaStream_t or NULL. */
LVBH_API int  lvbh_copy_to_host(lvbh_ctx *ctx, void *dst_host, const void *src_device, size_t bytes,
                                void *stream);

/* Bytes of device scratch a build of `num_tris` triangles needs beyond its inputs/outputs. */
LVBH_API size_t lvbh_scratch_bytes(uint32_t num_tris);

/* Text of the last error on this context (never NULL). */
LVBH_API const char *lvbh_last_error(const lvbh_ctx *ctx);
/* Library version string. */
LVBH_API const char *lvbh_version(void);

/* ---- build server: continuous batching under an HBM budget --------------------------
 * No counterpart in the reference, whose build() is one awaited call per scene
 * (scripts/bvh/build-bvh.js:12-66, scripts/main.js:88).  A server owns a scheduler thread,
 * `slots` build contexts each on its own stream, and one device reservation of `hbm_budget`
 * bytes that holds the contexts' scratch, each slot's staged input and every result until the
 * client releases it.  Submitted requests queue; whenever a slot is free, the scheduler takes
 * the queued requests in arrival order (up to max_batch_tris triangles and max_batch_reqs
 * requests, and what the free result memory admits), copies their triangles into the slot's
 * input, and runs one lvbh_build_batched over them.  Requests arriving while batches are on
 * the GPU are coalesced into the next batch and their copies and kernels overlap the batches
 * in flight.  Each result is bit-identical to lvbh_build_soup of the request alone. */
typedef struct lvbh_server lvbh_server;

typedef struct lvbh_server_config {
    int      device;          /* CUDA device ordinal; -1 = the calling thread's current device */
    uint32_t slots;           /* batches in flight at once (0 = 3) */
    uint64_t hbm_budget;      /* device bytes for scratch, staged inputs and results (0 = 96 GB) */
    uint32_t max_batch_tris;  /* largest batch and largest request (0 = 2^24) */
    uint32_t max_batch_reqs;  /* most requests per batch (0 = 4096) */
    uint32_t max_requests;    /* queued + in flight + unreleased (0 = 2^20); beyond: LVBH_EBUSY */
    uint32_t pad;
    uint64_t reserved[4];     /* must be zero */
} lvbh_server_config;

typedef struct lvbh_request_info {
    int      status;      /* LVBH_OK, LVBH_EBUSY while not finished, else the build's error status */
    uint32_t num_tris;
    uint32_t batch_reqs;  /* requests in the batch that built it */
    uint32_t batch_tris;  /* triangles in that batch */
    double   queued_ms;   /* submit -> its batch was launched */
    double   latency_ms;  /* submit -> its batch finished on the device */
} lvbh_request_info;

typedef struct lvbh_server_stats {
    uint64_t submitted, completed, failed, batches, tris_built;
    uint64_t budget_bytes;    /* the reservation */
    uint64_t result_bytes;    /* part of it available to results */
    uint64_t bytes_in_use;    /* results held now */
    uint64_t peak_bytes;      /* most results held at once */
    uint64_t admission_waits; /* times a queued batch waited for result memory */
    uint32_t max_batch_seen;  /* most requests coalesced into one batch */
    uint32_t pad;
} lvbh_server_stats;

LVBH_API int  lvbh_server_create(lvbh_server **srv, const lvbh_server_config *cfg);
/* Finishes the queued and in-flight requests, then frees everything (results included). */
LVBH_API void lvbh_server_destroy(lvbh_server *srv);
/* Queues one build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS).  tri: 12 floats per triangle, device
 * memory or (LVBH_INPUT_HOST) host memory - pinned host memory lets the copy overlap other
 * batches; either must stay valid until the request has finished.  model_bounds: 6 host
 * floats or NULL (reduce on the device), copied inside the call.  Returns LVBH_EINVAL for
 * num_tris > max_batch_tris, LVBH_ENOMEM when the request could never fit the result memory,
 * LVBH_EBUSY when max_requests are held. */
LVBH_API int  lvbh_submit(lvbh_server *srv, const float *tri, uint32_t num_tris,
                          const float *model_bounds, uint32_t flags, uint64_t *ticket);
/* LVBH_EBUSY while the request is not finished; then its status, with *out (device pointers
 * into the server's memory, valid until lvbh_request_release) and *info filled.  out and info
 * may be NULL.  LVBH_EINVAL for an unknown ticket. */
LVBH_API int  lvbh_poll(lvbh_server *srv, uint64_t ticket, lvbh_result *out, lvbh_request_info *info);
/* As lvbh_poll, waiting up to timeout_ms (< 0: without limit) for the request to finish. */
LVBH_API int  lvbh_wait(lvbh_server *srv, uint64_t ticket, int timeout_ms, lvbh_result *out,
                        lvbh_request_info *info);
/* Returns a finished request's result memory to the server (LVBH_EBUSY if not finished). */
LVBH_API int  lvbh_request_release(lvbh_server *srv, uint64_t ticket);
LVBH_API int  lvbh_server_stats_get(lvbh_server *srv, lvbh_server_stats *out);
LVBH_API const char *lvbh_server_last_error(const lvbh_server *srv);

/* ---- allocation-free sort -------------------------------------------------------------
 * No counterpart in the reference.  The build's stable radix sort of (key, index), for callers
 * that cannot allocate device memory when they need it: a render or serving loop that must not
 * stall (cudaMalloc / cudaFree synchronise the device), a process whose whole memory budget is
 * already reserved by its own pool, or a plugin host that owns every device allocation.
 *   keys_in   num_keys uint32 keys, device memory (not modified)
 *   keys_out  num_keys sorted keys (may be keys_in itself: in place); perm_out num_keys input
 *             indices (ties keep input order)
 *   stream    cudaStream_t or NULL; the call returns once the sort has finished
 * All other memory (ping-pong keys and values, histograms, look-back words, error word) is one
 * file-scope device array inside the library, sized for LVBH_NOALLOC_MAX_KEYS keys (about
 * 9.6 MB, held by every GPU that loads the library until the process exits); larger inputs are
 * rejected with LVBH_ERANGE before any GPU work.  The first call on each device looks up that
 * array's device address (cudaGetSymbolAddress, with the device current); make it before any
 * stream capture.  Calls share the array: two calls that overlap on the GPU (unordered
 * streams, or threads) race.  Calls no cudaMalloc, cudaFree or allocating routine.
 * Returns LVBH_OK, LVBH_ERANGE, LVBH_EINVAL (NULL pointer), LVBH_ETIMEOUT (a look-back wait
 * gave up), LVBH_EDEVICE (any other device-side error, e.g. a scatter target out of range when
 * calls overlap; the outputs are then incomplete) or LVBH_ECUDA. */
#define LVBH_NOALLOC_MAX_KEYS ((uint32_t)1 << 20)
LVBH_API int  lvbh_sort_pairs_noalloc(const uint32_t *keys_in, uint32_t num_keys,
                                      uint32_t *keys_out, uint32_t *perm_out, void *stream);

/* ---- validation consumer: closest-hit traversal ------------------------------------
 * Restates intersect_bvh / aabb_intersect / tri_intersect of scripts/pathtracer/pathtracer.js
 * (:495-584, :621-628, :587-619) over a built tree and returns per ray the hit triangle's
 * sorted position (-1 = miss), the hit distance t (-1 = miss, as the reference returns) and
 * the deepest stack the ray used.  rays: 8 floats per ray {ox,oy,oz,pad,dx,dy,dz,pad},
 * device memory. */
LVBH_API int  lvbh_trace(lvbh_ctx *ctx, const void *nodes, const void *tris, uint32_t num_tris,
                const float *rays, uint32_t num_rays, int32_t *hit_prim, float *hit_t,
                uint32_t *max_stack, void *stream);

/* lvbh_trace over the indexed leaf format (lvbh_build_mesh): leaf i's vertices are
 * verts4[leaf_idx3[3i..3i+2]] (16-byte rows, device memory); results equal lvbh_trace's over
 * the same triangles as a soup.  Indices >= num_verts read row 0. */
LVBH_API int  lvbh_trace_mesh(lvbh_ctx *ctx, const void *nodes, const uint32_t *leaf_idx3,
                const float *verts4, uint32_t num_verts, uint32_t num_tris, const float *rays,
                uint32_t num_rays, int32_t *hit_prim, float *hit_t, uint32_t *max_stack, void *stream);

/* ---- consumer: one path-trace bounce per pixel -------------------------------------
 * Replaces sample() (scripts/pathtracer/pathtracer.js:360-392): the compute shader main /
 * ptStep (:630-713) advances every pixel's path by one bounce - camera ray for a new path,
 * closest hit through the tree (:495-628), Lambertian bounce with Russian roulette after three
 * bounces, radiance 8 x throughput on a miss - over four rgba32f state images kept as device
 * buffers (no textures, no swapchain): planes o (origin, seed), d (direction, bounce count),
 * t (accumulated radiance, sample count), b (throughput, 1), each width x height float4, pixel
 * (x, y) at y * width + x.  state_in is read unless frame->rst is non-zero (the reset that
 * starts every path over); state_out receives the next state (ping-pong the two, as the
 * reference does).  The shader's implementation-defined functions are fixed: normalize(v) =
 * v / sqrt(dot(v, v)), sin / cos by a Cody-Waite reduction and Taylor polynomials (2 ulp),
 * pow(.3, 2.2) and sin(fov / 2) the nearest floats, aspect = (float)(width / height).
 * nodes / tris: a built tree (lvbh_result), device memory.  Returns LVBH_OK, LVBH_EINVAL or
 * LVBH_ECUDA; the call returns once the bounce has finished. */
typedef struct lvbh_pt_frame {
    float pos[3];  /* camera position (the uniform buffer's pos) */
    float rst;     /* non-zero: every path starts over (the uniform buffer's rst) */
    float lat[3];  /* look-at point */
    float pad;
} lvbh_pt_frame;
LVBH_API int  lvbh_pt_sample(lvbh_ctx *ctx, const void *nodes, const void *tris, uint32_t num_tris,
                             const float *state_in, float *state_out, uint32_t width, uint32_t height,
                             const lvbh_pt_frame *frame, void *stream);

/* ---- producer: OBJ text -> TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS ------------------------
 * Replaces parseObj(file) (scripts/obj/parse-obj.js:3-88) and the OBJFile parser it calls
 * (scripts/obj/obj-file-parser.js:19-193), the step main.js:72-73 runs before build().  The
 * text (UTF-8 bytes, as FileReader.readAsText reads them) is parsed on the GPU with the
 * reference's results: model 0's faces fan-triangulated, y and z swapped, as 12 float32 per
 * triangle with pad 3.1415, two floor triangles appended; bounds6 the six doubles of BOUNDS
 * (min xyz, max xyz) with Math.min / Math.max semantics.
 *   text      `bytes` bytes, device memory, or host memory with LVBH_INPUT_HOST
 *   bytes     at most LVBH_OBJ_MAX_BYTES
 *   tri_out   receives a device pointer to *num_tris x 12 floats, owned by ctx and valid until
 *             the next lvbh_parse_obj on ctx or lvbh_destroy (pass it to lvbh_build_soup)
 *   err_line  where the reference throws: the 1-based line of the statement it rejects, or 0
 *             for a failure found after parsing (no model; a face index naming no vertex)
 *   stream    cudaStream_t or NULL; the call returns once the soup is complete
 * Returns LVBH_OK, LVBH_EPARSE (with *err_line, and the reason in lvbh_last_error),
 * LVBH_EINVAL (NULL pointer, size beyond LVBH_OBJ_MAX_BYTES), LVBH_ENOMEM or LVBH_ECUDA. */
#define LVBH_OBJ_MAX_BYTES ((uint64_t)0xFFFFFE00u)
LVBH_API int  lvbh_parse_obj(lvbh_ctx *ctx, const char *text, uint64_t bytes, uint32_t flags,
                             const float **tri_out, uint32_t *num_tris, double *bounds6,
                             uint64_t *err_line, void *stream);

/* ---- test hook: a device wait that runs out --------------------------------------------
 * No counterpart in the reference (its shaders spin without a bound).  For tests of the
 * bounded waits: on this context, sort tile `stall_tile` (0-based, in the order tiles start) of
 * every decoupled look-back sort pass (the batched build's) publishes no counts, so the tiles
 * after it in its mesh wait until their bound runs out; the build then returns LVBH_ETIMEOUT
 * and builds no tree from the unfinished sort.  spin_cycles, when not 0, replaces the bound
 * (about 2e9 clock cycles, a second).  lvbh_test_stall_lookback(ctx, UINT32_MAX, 0) restores
 * normal builds.  Finishes a pending LVBH_ASYNC build first (returning its status if it
 * failed).  Returns LVBH_OK, LVBH_EINVAL or LVBH_ECUDA. */
LVBH_API int  lvbh_test_stall_lookback(lvbh_ctx *ctx, uint32_t stall_tile, uint32_t spin_cycles);

#ifdef __cplusplus
}
#endif
#endif /* LVBH_H */
