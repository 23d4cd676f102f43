// emit.cu - K3: radix tree emission, leaf gather, triangle rearrange and bottom-up refit
// (sm_100a).
//
// Produces what the reference computes in three kernels: compute_radix_tree_pointers
// (scripts/bvh/kernels/radix-tree.js:137-238, parent links), bvh_upward_pass
// (scripts/bvh/kernels/bvh-up-pass.js:200-280, node boxes and child links) and
// rearrange_triangles (scripts/bvh/kernels/rearrange.js:162-169).
//
// Tree.  With d[k] = delta(k, k+1) (common-prefix length of adjacent sorted keys, index
// tie-break, -1 past either end), the Karras radix tree is the Cartesian tree of d: the node
// whose split is s covers [L, R], where L-1 and R are the nearest positions left and right of
// s with a smaller d.  A node [L, R] is the LEFT child of split R when d[R] > d[L-1], else the
// RIGHT child of split L-1 (adjacent d values always differ), so its Karras index is R or L
// (0 for the root) - exactly the numbering compute_child_index produces - and its parent
// follows from its own range alone.  The tree is therefore built bottom-up with the boxes:
// every leaf climbs; at each split the first child to arrive parks, the second merges both
// into the parent's record and climbs on.  No per-node binary search, N-1 box unions.
//
// Passes.
//   K3b (k_tree_climb)   blocks of 256 sorted leaves in shared memory, a persistent grid that
//                        prefetches the next blocks: leaf k's triangle perm[k] arrives with
//                        three others by one TMA gather of four 48-byte rows, goes to the
//                        output soup at k and is reduced to its
//                        box (exact-zero components nudged by 1e-8 as bvh-up-pass.js:209-210
//                        does).  The climb runs in steps:
//                        the items still climbing after a step are compacted into a queue, so
//                        warps stay full while the number of items shrinks.  Parking and
//                        merging use an arrival mask per split (shared-memory atomics) and
//                        parked items in shared memory; records go straight to the node
//                        buffer, parent links are staged and written coalesced.  An item
//                        whose parent split lies outside the block, or whose sibling never
//                        arrives (the parent straddles the block boundary), leaves as an
//                        "open item" (at most 2 x 64 per block: they hang off the two boundary
//                        paths of a tree at most 64 deep).
//   K3c (k_top_group)    the nodes that straddle blocks (~3 % of them), built bottom-up from
//                        the open items: per group of blocks in shared memory, then with
//                        arrival words in global memory (see below).
#include <cstring>
#include <cuda.h>  // CUtensorMap
#include <cudaTypedefs.h>
#include <type_traits>

#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

// Tree-pass geometry: blocks of 2^LOG sorted leaves (one thread each), resident CTAs per SM
// of the persistent grid.  The plain build uses LOG = 8; a batched build may pick LOG = 7.
template <int LOG>
struct TreeGeo {
    static constexpr int EB = 1 << LOG;
    static constexpr int kCtasPerSm = LOG == 8 ? 4 : 8;
    static_assert(2 * LOG + 14 <= 32, "packed item ranges");
    // packed local range and end separators of a climbing item:
    // l | r << LOG | (d[l-1] + 1) << 2 LOG | (d[r] + 1) << 2 LOG + 7   (d + 1 <= 64)
    static __device__ __forceinline__ uint32_t pack(int l, int r, int dl, int dr) {
        return (uint32_t)l | ((uint32_t)r << LOG) | ((uint32_t)(dl + 1) << (2 * LOG)) |
               ((uint32_t)(dr + 1) << (2 * LOG + 7));
    }
    static __device__ __forceinline__ int rl(uint32_t p) { return (int)(p & (EB - 1)); }
    static __device__ __forceinline__ int rr(uint32_t p) { return (int)((p >> LOG) & (EB - 1)); }
    static __device__ __forceinline__ int rdl(uint32_t p) { return (int)((p >> (2 * LOG)) & 127u) - 1; }
    static __device__ __forceinline__ int rdr(uint32_t p) { return (int)(p >> (2 * LOG + 7)) - 1; }
};
constexpr int kTopLanes = 8;                   // K3c threads per block of K3b
constexpr int kFreeClimb = 64;                 // K3b items left when compaction stops

// Where a block of EB sorted leaves lives.  A batched build is a list of segments (meshes)
// laid end to end; every block lies inside one segment and every index a kernel works with
// is local to that segment (the plain build is the one-segment case).
struct Span {
    size_t start;  // the segment's first position in the batch
    int n;         // the segment's triangle count
    int b0;        // the block's first leaf within the segment
};

template <int LOG>
struct OneSeg {
    static constexpr int EB = 1 << LOG;
    int n;
    __device__ __forceinline__ int blocks() const { return (n + EB - 1) / EB; }
    __device__ __forceinline__ Span span(int blk) const { return Span{0, n, blk * EB}; }
    __device__ __forceinline__ size_t item_base(int blk, int cap) const { return (size_t)blk * cap; }
};

template <int LOG>
struct ManySegs {
    static constexpr int EB = 1 << LOG;
    const SegRow *rows;       // num_segs + 1 rows
    const uint32_t *blk_seg;  // segment of each block
    int nblk;
    __device__ __forceinline__ int blocks() const { return nblk; }
    __device__ __forceinline__ Span span(int blk) const {
        const uint32_t sg = __ldg(blk_seg + blk);
        const uint32_t t0 = __ldg(&rows[sg].tri), t1 = __ldg(&rows[sg + 1].tri);
        const int first = (int)__ldg(&rows[sg].blk);
        return Span{t0, (int)(t1 - t0), (blk - first) * EB};
    }
    __device__ __forceinline__ size_t item_base(int blk, int cap) const { return (size_t)blk * cap; }
};

// K3b shared memory.  A climbing item is two float4: box min + link (node index, or
// -(leaf + 1)), box max + its packed local range and end separators (TreeGeo::pack).
// Where the tree pass gets its leaves.  SoupLeaves: leaf t of a block is triangle perm[b0 + t]
// of the 48-byte soup, copied to the output soup.  MeshLeaves (the indexed leaf format): leaf t
// is the sorted triangle b0 + t, whose three vertex indices are already in sorted order
// (sidx, written by the leaf-index pass) and whose vertices are 16-byte rows of a vertex
// buffer; nothing is copied.
struct SoupLeaves {
    static constexpr bool kMesh = false;
    const float4 *tri;
    const uint32_t *perm;
    float4 *otri;
};
struct MeshLeaves {
    static constexpr bool kMesh = true;
    const float4 *verts;
    const uint32_t *sidx;
    uint32_t nverts;
};

// The gathered triangles of this block and the next: buffer b holds leaves 4g .. 4g + 3 in
// slot[b][g], four 48-byte rows (float4 0..11, one tensor gather each) in a 256-byte slot, so
// that every gather's destination starts on a 128-byte boundary.  The slots' last 64 bytes
// (float4 12..15), which no copy writes, hold the step queues: [queue][min/max][item] of the
// items of the current and the next step (a step after the first has at most EB / 2: every
// merge takes two items), entry f = (queue * 2 + min/max) * EB / 2 + item at flat slot f / 4,
// float4 12 + f % 4.
template <int EB, int PROW>
struct ClimbSmem {
    float4 slot[2][EB / 4][16];
    float4 pend[2][2][EB];  // [side][min/max][split] the child parked at each split.  Split
                            // index innermost keeps the 16-byte accesses of random splits off
                            // each other's banks.
    uint32_t key[EB + 2];   // keys of leaves b0-1 .. b0+EB
    uint32_t mask[EB];      // arrivals at each split: bit 0 left child, bit 1 right child
    int par[2 * EB];        // parent of internal node b0 + j at j, of leaf b0 + j at EB + j
                            // (-1 = not set here)
    uint32_t prow[PROW];    // soup, one segment: the rows of the block two ahead, staged for its gathers
    Span sp2[2];            // soup: the span of the block two ahead of an iteration on buffer b
    int cnt[3];             // item counters, rotating over the steps
    int open[2];            // open items emitted, by buffer parity (a block's and the next's)
    uint64_t bar[2];        // completion of the gathers into slot[0] / slot[1]
};

// Whether a tree pass issues its soup gathers late (see issue_next in k_tree_climb) and its
// shared-memory layout.
template <int LOG, class Segs, class Leaves>
struct TreeLayout {
    static constexpr bool kLate = !Leaves::kMesh && std::is_same<Segs, OneSeg<LOG>>::value;
    using Smem = ClimbSmem<(1 << LOG), kLate ? (1 << LOG) : 1>;
};

// K3b: leaf gather, rearrange and the tree over blocks of EB sorted leaves (see the pass list
// above).  Leaf t of a block gathers triangle perm[b0 + t]: its index is loaded three blocks
// ahead, its 48-byte row is copied into shared memory two blocks ahead (with those of leaves
// t+1..t+3 by one tile::gather4 copy through `soup_map`, the soup as a tensor of 12-float
// rows, completing on the buffer's mbarrier; no registers held meanwhile), then written to the
// output soup and reduced to the leaf box.  A mesh leaf's three 16-byte vertex rows (mostly L2
// hits) come by cp.async instead (soup_map unused).
template <int LOG, class Segs, class Leaves = SoupLeaves>
__global__ void __launch_bounds__(TreeGeo<LOG>::EB, TreeGeo<LOG>::kCtasPerSm) k_tree_climb(Segs segs,
                                                    const uint32_t *__restrict__ keys_all,
                                                    Leaves lv,
                                                    float4 *nodes_all, int32_t *parents_all,
                                                    OpenItem *out_items, uint32_t *out_counts,
                                                    Control *ctl, const __grid_constant__ CUtensorMap soup_map) {
    using G = TreeGeo<LOG>;
    constexpr int EB = G::EB;
    constexpr int kFree = kFreeClimb < EB / 2 ? kFreeClimb : EB / 2;  // the free climb leaves threads
                                                                     // EB / 2 .. 3 EB / 4 - 1 idle
    // the soup gathers of a one-segment build issued late, by threads the free climb leaves idle
    // (a batch keeps them in the refill: its extra state spilled there, 13.6 -> 14.1 ms a batch)
    using Layout = TreeLayout<LOG, Segs, Leaves>;
    constexpr bool kLate = Layout::kLate;
    extern __shared__ __align__(16) unsigned char smem[];
    // the layout from the first 128-byte boundary (the launch adds 128 bytes of slack)
    typename Layout::Smem &S =
        *reinterpret_cast<typename Layout::Smem *>(smem + ((128u - (smem_addr(smem) & 127u)) & 127u));
    // leaf t's three rows in buffer b; entry f of the step queues (see ClimbSmem)
    auto tri_row = [&](int b, int x) -> float4 * { return &S.slot[b][x >> 2][(x & 3) * 3]; };
    auto qent = [&](int f) -> float4 & { return (&S.slot[0][0][0])[(f >> 2) * 16 + 12 + (f & 3)]; };
    const int t = threadIdx.x, lane = t & 31;
    chain_wait();
    // a sort whose look-back gave up left unsorted keys: build nothing from them (uniform)
    if (ld_relaxed_gpu(&ctl->err) & ERR_LOOKBACK_TIMEOUT) return;
    const int nblk = segs.blocks();
    const uint32_t lt = lanemask_lt();

    // Leaves come in three steps ahead of their block: this thread's permutation entry (its three
    // vertex indices for a mesh) three blocks ahead, its triangle copied into slot[] two blocks
    // ahead, its key one block ahead.  Two buffers, slot[0] and slot[1], serve the copies two
    // blocks ahead: a block's buffer is refilled once its own leaf phase has read it (right after
    // it, or for a one-segment soup during the block's free climb), so the copies of two blocks
    // are in flight while a block climbs.
    uint32_t pa = 0, pb = 0, pc = 0;
    auto fetch_perm = [&](int blk) {
        const Span sp = segs.span(blk);
        if (sp.b0 + t < sp.n) {
            if constexpr (Leaves::kMesh) {
                const uint32_t *r = lv.sidx + 3ull * (sp.start + sp.b0 + t);
                pa = __ldg(r);
                pb = __ldg(r + 1);
                pc = __ldg(r + 2);
            } else {
                pa = __ldg(lv.perm + sp.start + sp.b0 + t);
            }
        }
    };
    bool bad_perm = false;
    // The block's triangles into slot[buf].  Soup: thread 4g issues one tile::gather4 copy of
    // leaves 4g .. 4g+3 (rows sp.start + perm) on the buffer's mbarrier, whose phase expects 192
    // bytes per group of four of the block (thread 0's arrival is its only one); a leaf past the
    // segment in the last group repeats its group's first row (read, never used).  The copy
    // engine takes about one small copy per 11 to 17 cycles per SM, which one 48-byte copy per
    // leaf kept saturated; with four rows a copy and the tensor map's 64-byte L2 fills a random
    // gather of 16.7 M rows takes 0.55 ms against 0.67 (B200; DRAM reads 154 -> 98 B per row).
    // Mesh: the vertex rows (mostly in L2) by cp.async, one commit group per thread and block.
    auto fetch_tri = [&](int blk, int buf) {
        const Span sp = segs.span(blk);
        const int b0 = sp.b0, n = sp.n, k = b0 + t;
        if constexpr (Leaves::kMesh) {
            if (k < n) {
                // an index past the vertex buffer was reported by the Morton pass; read row 0
                const uint32_t nv = lv.nverts;
                float4 *d = tri_row(buf, t);
                cp_async16(d, lv.verts + (pa < nv ? pa : 0u));
                cp_async16(d + 1, lv.verts + (pb < nv ? pb : 0u));
                cp_async16(d + 2, lv.verts + (pc < nv ? pc : 0u));
            }
            cp_async_commit();
        } else {
            if (t == 0) mbar_arrive_tx(&S.bar[buf], 192u * (uint32_t)((min(EB, n - b0) + 3) / 4));
            uint32_t row = 0;
            if (k < n) {
                uint32_t ti = pa;
                if (ti >= (uint32_t)n) { bad_perm = true; ti = 0; }
                row = (uint32_t)(sp.start + ti);
            }
            const uint32_t r1 = __shfl_down_sync(0xFFFFFFFFu, row, 1), r2 = __shfl_down_sync(0xFFFFFFFFu, row, 2),
                           r3 = __shfl_down_sync(0xFFFFFFFFu, row, 3);
            if ((t & 3) == 0 && k < n)
                gather4_g2s(tri_row(buf, t), &soup_map, row, k + 1 < n ? r1 : row, k + 2 < n ? r2 : row,
                            k + 3 < n ? r3 : row, &S.bar[buf]);
        }
    };
    // one block ahead: its span, this thread's key, the keys on either side of the block
    Span nsp{0, 0, 0};
    uint32_t nk = 0, nk_lo = 0, nk_hi = 0;
    auto fetch_keys = [&](int blk) {
        nsp = segs.span(blk);
        const uint32_t *keys = keys_all + nsp.start;
        const int b0 = nsp.b0, n = nsp.n, k = b0 + t;
        if (k < n) nk = __ldg(keys + k);
        if (t == 0) nk_lo = b0 > 0 ? __ldg(keys + b0 - 1) : 0u;
        if (t == EB - 1) nk_hi = (b0 + EB < n) ? __ldg(keys + b0 + EB) : 0u;
    };
    const int grid = (int)gridDim.x;
    // after every thread has read slot[buf] (a barrier between): load the permutation three
    // ahead and, for mesh leaves, refill the buffer with the block two ahead
    auto refill = [&](int blk, int buf) {
        if (blk + 2 * grid >= nblk) return;
        if constexpr (!kLate) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // reads above, copies below
            fetch_tri(blk + 2 * grid, buf);
        }
        if (blk + 3 * grid < nblk) {
            fetch_perm(blk + 3 * grid);
            if (kLate && t == 0) S.sp2[buf ^ 1] = segs.span(blk + 3 * grid);  // the next iteration's
        }
    };
    // Soup: the block two ahead's gathers into slot[buf] (read by now), group g of it (leaves
    // 4g .. 4g+3, rows staged in prow).  Issued by threads that the free climb leaves idle: the
    // 64 copies of a block queue on the copy engine for ~2,300 cycles, a stall that delayed the
    // whole block's first climb step when every fourth thread issued them after the leaf phase
    // (tree pass 0.90 -> 0.886 ms on 16.7 M).
    auto issue_next = [&](int blk, int buf, int g) {
        if (blk + 2 * grid >= nblk) return;
        const Span s2 = S.sp2[buf];
        const int m2 = min(EB, s2.n - s2.b0), ng = (m2 + 3) / 4;
        if (g == 0) mbar_arrive_tx(&S.bar[buf], 192u * (uint32_t)ng);
        if (g < ng) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // reads above, copies below
            const int x = 4 * g;  // a leaf past the segment repeats its group's first row
            const uint32_t r0 = S.prow[x];
            gather4_g2s(&S.slot[buf][g][0], &soup_map, r0, x + 1 < m2 ? S.prow[x + 1] : r0,
                        x + 2 < m2 ? S.prow[x + 2] : r0, x + 3 < m2 ? S.prow[x + 3] : r0, &S.bar[buf]);
        }
    };
    int buf = 0;
    uint32_t phase = 0;  // bit b: parity of the next phase of S.bar[b] (uniform over the block)
    bool copy_timeout = false;
    if (t < 2) mbar_init(&S.bar[t], 1);
    if (t < 2) S.open[t] = 0;
    if (kLate && t == 0 && (int)blockIdx.x + 2 * grid < nblk) S.sp2[0] = segs.span(blockIdx.x + 2 * grid);
    mbar_init_fence();
    __syncthreads();
    if ((int)blockIdx.x < nblk) {
        fetch_perm(blockIdx.x);
        fetch_tri(blockIdx.x, 0);
        fetch_keys(blockIdx.x);
        if ((int)blockIdx.x + grid < nblk) {
            fetch_perm(blockIdx.x + grid);
            fetch_tri(blockIdx.x + grid, 1);
            if ((int)blockIdx.x + 2 * grid < nblk) fetch_perm(blockIdx.x + 2 * grid);
        }
    }

    // Thread 0, after a barrier that follows the previous block's emissions: that block's count
    // of open items, and its counter cleared for the next block (the counters alternate with the
    // buffers).  No barrier ends a block: every shared word a thread reads after the climb (its
    // own mask, links and parked pair) it resets itself at the next block's start, and the next
    // block touches anyone else's only after its leaf barrier (a barrier at the end of each
    // block cost the pass 0.852 -> 0.890 ms on 16.7 M).
    auto settle_prev = [&](int blk, int buf) {
        if (blk - grid >= (int)blockIdx.x) {
            const int o = S.open[buf ^ 1];
            out_counts[blk - grid] = (uint32_t)min(o, kOpenCap);
            if (o > kOpenCap) atomicOr(&ctl->err, ERR_CLIMB);
        }
        S.open[buf ^ 1] = 0;
    };
    int last = -1, last_buf = 0;
    for (int blk = blockIdx.x; blk < nblk; blk += grid, buf ^= 1) {
        last = blk;
        last_buf = buf;
        const Span sp = nsp;
        const int b0 = sp.b0, n = sp.n;
        float4 *nodes = nodes_all + 4ull * sp.start;
        int32_t *parents = parents_all + 2ull * sp.start;
        const int m = min(EB, n - b0);
        const int k = b0 + t;
        const bool active = t < m;
        S.key[t + 1] = active ? nk : 0u;
        if (t == 0) S.key[0] = nk_lo;
        if (t == EB - 1) S.key[EB + 1] = nk_hi;
        S.mask[t] = 0;
        S.par[t] = -1;
        S.par[EB + t] = -1;
        if (t < 3) S.cnt[t] = 0;
        // this leaf's triangle: to the output soup, and its box (exact-zero components nudged
        // by 1e-8 as bvh-up-pass.js:209-210 does)
        if constexpr (Leaves::kMesh) {
            // the next block's group may still be in flight (the newest one), not this one's
            if (blk + grid < nblk) asm volatile("cp.async.wait_group 1;" ::: "memory");
            else cp_async_wait_all();
        } else {
            if (!mbar_wait(&S.bar[buf], (phase >> buf) & 1u)) copy_timeout = true;
            phase ^= 1u << buf;
        }
        float4 leaf_lo = make_float4(0.f, 0.f, 0.f, __int_as_float(-(k + 1)));
        float4 leaf_hi0 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (active) {
            const float4 *tr = tri_row(buf, t);
            const float4 a = tr[0], b = tr[1], c = tr[2];
            if constexpr (!Leaves::kMesh) {
                float4 *dst = lv.otri + 3ull * (sp.start + k);
                st_stream(dst, a);
                st_stream(dst + 1, b);
                st_stream(dst + 2, c);
            }
            float nx = fminf(a.x, fminf(b.x, c.x)), ny = fminf(a.y, fminf(b.y, c.y)), nz = fminf(a.z, fminf(b.z, c.z));
            float xx = fmaxf(a.x, fmaxf(b.x, c.x)), xy = fmaxf(a.y, fmaxf(b.y, c.y)), xz = fmaxf(a.z, fmaxf(b.z, c.z));
            nx = nx == 0.0f ? -1e-8f : nx; ny = ny == 0.0f ? -1e-8f : ny; nz = nz == 0.0f ? -1e-8f : nz;
            xx = xx == 0.0f ? 1e-8f : xx;  xy = xy == 0.0f ? 1e-8f : xy;  xz = xz == 0.0f ? 1e-8f : xz;
            leaf_lo = make_float4(nx, ny, nz, __int_as_float(-(k + 1)));
            leaf_hi0 = make_float4(xx, xy, xz, 0.f);
        }
        if (blk + grid < nblk) fetch_keys(blk + grid);
        if constexpr (kLate) {  // this thread's row of the block two ahead
            if (blk + 2 * grid < nblk) {
                const Span s2 = S.sp2[buf];
                uint32_t row = 0;
                if (s2.b0 + t < s2.n) {
                    uint32_t ti = pa;
                    if (ti >= (uint32_t)s2.n) { bad_perm = true; ti = 0; }
                    row = (uint32_t)(s2.start + ti);
                }
                S.prow[t] = row;
            }
        }
        if (n == 1) {  // one leaf, one arrival at node 0: left slot only, f_1 = 1
            if (t == 0) {
                nodes[0] = make_float4(leaf_lo.x, leaf_lo.y, leaf_lo.z, __int_as_float(-1));
                nodes[1] = make_float4(leaf_hi0.x, leaf_hi0.y, leaf_hi0.z, __int_as_float(1));
                nodes[2] = make_float4(0.f, 0.f, 0.f, 0.f);
                nodes[3] = make_float4(0.f, 0.f, 0.f, 0.f);
                parents[0] = 0;
                parents[1] = 0;
                out_counts[blk] = 0;
            }
            // uniform across the block; no other thread reads what this one wrote.  The barrier
            // keeps every thread's wait on this buffer's phase ahead of its next arming.
            __syncthreads();
            if (t == 0) settle_prev(blk, buf);
            refill(blk, buf);
            if constexpr (kLate)
                if (t < EB / 4) issue_next(blk, buf, t);
            continue;
        }
        if (k == 0) {  // the root has no parent; slot N-1 and record N-1 stay zero
            parents[0] = 0;
            parents[n - 1] = 0;
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            float4 *last = nodes + 4ull * (n - 1);
            last[0] = z; last[1] = z; last[2] = z; last[3] = z;
        }
        __syncthreads();  // every thread has waited on and read slot[buf]: it may be refilled
        if (t == 0) settle_prev(blk, buf);
        refill(blk, buf);
        auto dval = [&](int x) -> int {  // d of split b0 + x, x in [-1, EB - 1]
            const int g = b0 + x;
            if (g < 0 || g >= n - 1) return -1;
            const uint32_t a = S.key[x + 1], b = S.key[x + 2];
            return a != b ? __clz(a ^ b) : 32 + __clz(g ^ (g + 1));
        };
        OpenItem *out = out_items + (size_t)blk * kOpenCap;
        auto emit = [&](float4 lo, float4 hi) {  // an item leaves the block for K3c
            const uint32_t pk = __float_as_uint(hi.w);
            OpenItem it;
            it.lo = lo;
            it.hi = make_float4(hi.x, hi.y, hi.z, __int_as_float(G::rdr(pk)));
            it.xl = b0 + G::rl(pk);
            it.xr = b0 + G::rr(pk);
            it.pad0 = G::rdl(pk);
            it.pad1 = 0;
            const int at = atomicAdd(&S.open[buf], 1);
            if (at < kOpenCap) out[at] = it;
            else atomicOr(&ctl->err, ERR_CLIMB);
        };
        // One step of an item: leave the block, park at its parent split, or merge with the
        // parked sibling into the parent (returned in nlo/nhi, true unless it is the root).
        auto climb = [&](float4 lo, float4 hi, float4 &nlo, float4 &nhi) -> bool {
            const uint32_t pk = __float_as_uint(hi.w);
            const int l = G::rl(pk), r = G::rr(pk), dl = G::rdl(pk), dr = G::rdr(pk);
            const bool is_left = dr > dl;
            const int s = is_left ? r : l - 1;
            if (s < 0 || s > m - 2) {
                emit(lo, hi);
                return false;
            }
            const int side = is_left ? 0 : 1;
            S.pend[side][0][s] = lo;
            S.pend[side][1][s] = hi;
            if (atom_or_acq_rel_cta(&S.mask[s], 1u << side) == 0u) return false;  // first parks
            const float4 slo = S.pend[side ^ 1][0][s], shi = S.pend[side ^ 1][1][s];
            const uint32_t spk = __float_as_uint(shi.w);
            const int L = is_left ? l : G::rl(spk), R = is_left ? G::rr(spk) : r;
            const int ndl = is_left ? dl : G::rdl(spk), ndr = is_left ? G::rdr(spk) : dr;
            const bool root = (b0 + L == 0) && (b0 + R == n - 1);
            const int P = root ? 0 : (ndr > ndl ? b0 + R : b0 + L);
            // the record: this child in slot `side`, the sibling in the other (f_1 = 2, f_2 = 0)
            float4 *rc = nodes + 4ull * P;
            rc[2 * side] = lo;
            rc[2 * side + 1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(2 - 2 * side));
            rc[2 - 2 * side] = slo;
            rc[3 - 2 * side] = make_float4(shi.x, shi.y, shi.z, __int_as_float(2 * side));
            const int mref = __float_as_int(lo.w), sref = __float_as_int(slo.w);
            S.par[mref >= 0 ? mref - b0 : EB - 1 - b0 - mref] = P;
            S.par[sref >= 0 ? sref - b0 : EB - 1 - b0 - sref] = P;
            if (root) return false;
            nlo = make_float4(fminf(lo.x, slo.x), fminf(lo.y, slo.y), fminf(lo.z, slo.z), __int_as_float(P));
            nhi = make_float4(fmaxf(hi.x, shi.x), fmaxf(hi.y, shi.y), fmaxf(hi.z, shi.z),
                              __uint_as_float(G::pack(L, R, ndl, ndr)));
            return true;
        };
        // the items that climb on go to queue oq, counted in S.cnt[oc] (warp-aggregated)
        auto append = [&](bool cont, float4 nlo, float4 nhi, int oq, int oc) {
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, cont);
            int base = 0;
            if (lane == 0 && bal) base = atomicAdd(&S.cnt[oc], __popc(bal));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (cont) {
                const int at = base + __popc(bal & lt);
                qent((oq * 2) * (EB / 2) + at) = nlo;
                qent((oq * 2 + 1) * (EB / 2) + at) = nhi;
            }
        };

        // step 0: the leaves
        float4 nlo = make_float4(0.f, 0.f, 0.f, 0.f), nhi = nlo;
        bool cont = false;
        if (active)
            cont = climb(leaf_lo, make_float4(leaf_hi0.x, leaf_hi0.y, leaf_hi0.z,
                                              __uint_as_float(G::pack(t, t, dval(t - 1), dval(t)))),
                         nlo, nhi);
        append(cont, nlo, nhi, 0, 0);
        // later steps: the merged parents, compacted.  Once at most kFree items are left,
        // each takes one thread of the first warps and climbs on its own, item in registers,
        // without block barriers (the park / merge handshake works across warps).
        int cur = 0, c = 0;
        bool issued = false;  // the block two ahead's gathers (uniform)
        for (int guard = 0; guard < 2 * EB; ++guard) {
            __syncthreads();
            const int count = S.cnt[c];
            if (count <= kFree) {
                if (t < count) {
                    float4 lo = qent((cur * 2) * (EB / 2) + t), hi = qent((cur * 2 + 1) * (EB / 2) + t);
                    for (int g2 = 0; g2 < 2 * EB; ++g2) {
                        if (!climb(lo, hi, nlo, nhi)) break;
                        lo = nlo;
                        hi = nhi;
                    }
                } else if (kLate && t >= EB / 2 && t < EB / 2 + EB / 4) {
                    issue_next(blk, buf, t - EB / 2);  // count <= kFree <= EB / 2
                }
                issued = true;
                break;
            }
            const int nc = c == 2 ? 0 : c + 1, rc = nc == 2 ? 0 : nc + 1;
            cont = false;
            if (t < count) cont = climb(qent((cur * 2) * (EB / 2) + t), qent((cur * 2 + 1) * (EB / 2) + t), nlo, nhi);
            append(cont, nlo, nhi, cur ^ 1, nc);
            if (t == 0) S.cnt[rc] = 0;
            cur ^= 1;
            c = nc;
        }
        if (kLate && !issued && t < EB / 4) issue_next(blk, buf, t);
        __syncthreads();
        // a child parked at a split whose sibling never came: the parent straddles the block
        if (t < m - 1) {
            const uint32_t mk = S.mask[t];
            if (mk == 1u || mk == 2u) {
                const int side = mk == 1u ? 0 : 1;
                emit(S.pend[side][0][t], S.pend[side][1][t]);
            }
        }
        if (active) {  // the climb is over (barrier above): the staged links are final
            if (S.par[t] >= 0) parents[k] = S.par[t];
            if (S.par[EB + t] >= 0) parents[n + k] = S.par[EB + t];
        }
    }
    __syncthreads();  // the last block's open items are counted
    if (t == 0 && last >= 0) {
        const int o = S.open[last_buf];
        out_counts[last] = (uint32_t)min(o, kOpenCap);
        if (o > kOpenCap) atomicOr(&ctl->err, ERR_CLIMB);
    }
    if (bad_perm) atomicOr(&ctl->err, ERR_CLIMB);
    if (copy_timeout) atomicOr(&ctl->err, ERR_COPY_TIMEOUT);
}

// K3c, the arrival-word climb: each thread climbs an open item through the splits above it
// (k_top_group calls it for what leaves a group; k_emit_top, with kTopLanes threads per K3b
// block, over the blocks' items directly).  At a split the
// first arriving child parks its box, link and far range end in pend[] and its far end's
// separator in pend_d[], both at its own index (r when it is a left child, l when a right child -
// no two pending children ever share one), and exchanges the build's epoch into the split's
// arrival word with release-acquire semantics; the second, seeing the epoch already there,
// reads its sibling back,
// merges, and has the parent's range, both end separators and so its Karras index without
// touching the keys.  A completed record and its two parent links are stored after the next
// split's exchange, so that exchange's release waits for the parked rows only.
// Nothing waits, so the kernel cannot hang; climbs are bounded and every index is
// range-checked.  The epoch makes the arrival words reusable without clearing: a word left by
// an older build never equals the current epoch.
//
// One open item's climb through the splits above it with the arrival words, in a
// segment of n triangles whose node, parent, arrival and pending arrays start at the pointers
// given.  False if the climb broke off (a range inconsistent with the tree, or more levels than
// any tree has).
__device__ __forceinline__ bool top_climb(const OpenItem &it, int n, float4 *nodes, int32_t *parents, uint32_t *arrive,
                                          float4 *pend, uint8_t *pend_d, uint32_t epoch) {
    int l = it.xl, r = it.xr, ref = __float_as_int(it.lo.w);
    float nx = it.lo.x, ny = it.lo.y, nz = it.lo.z, xx = it.hi.x, xy = it.hi.y, xz = it.hi.z;
    int dl = it.pad0, dr = __float_as_int(it.hi.w);
    // the record completed at the previous split, stored after the next exchange
    bool have = false;
    float4 w0, w1, w2, w3;
    int wP = 0, wl = 0, wr = 0;
    auto flush = [&]() {
        if (!have) return;
        float4 *rc = nodes + 4ull * wP;
        rc[0] = w0; rc[1] = w1; rc[2] = w2; rc[3] = w3;
        parents[wl >= 0 ? wl : n - (wl + 1)] = wP;
        parents[wr >= 0 ? wr : n - (wr + 1)] = wP;
        have = false;
    };
    bool done = false;
    for (int level = 0; level < 160; ++level) {
        if (l == 0 && r == n - 1) { done = true; break; }  // root complete
        const bool is_left = dr > dl;
        const int s = is_left ? r : l - 1;
        if (s < 0 || s >= n - 1 || l < 0 || r >= n) break;
        const int own = is_left ? r : l, sib = is_left ? s + 1 : s;
        const float4 h0 = make_float4(nx, ny, nz, __int_as_float(ref));
        const float4 h1 = make_float4(xx, xy, xz, __int_as_float(is_left ? l : r));
        pend[2ull * own] = h0;
        pend[2ull * own + 1] = h1;
        pend_d[own] = (uint8_t)((is_left ? dl : dr) + 1);
        const bool first = atom_exch_acq_rel_gpu(arrive + s, epoch) != epoch;
        flush();
        if (first) { done = true; break; }  // the sibling completes the parent
        const float4 g0 = __ldcg(pend + 2ull * sib), g1 = __ldcg(pend + 2ull * sib + 1);
        const int gd = (int)__ldcg(pend_d + sib) - 1;
        const int sib_ref = __float_as_int(g0.w), sib_far = __float_as_int(g1.w);
        const int L = is_left ? l : sib_far, R = is_left ? sib_far : r;
        if (L < 0 || R >= n || L > l || R < r || sib_ref < -n || sib_ref >= n - 1) break;
        const float4 lo0 = is_left ? h0 : g0, lo1 = is_left ? h1 : g1;
        const float4 hi0 = is_left ? g0 : h0, hi1 = is_left ? g1 : h1;
        nx = fminf(nx, g0.x); ny = fminf(ny, g0.y); nz = fminf(nz, g0.z);
        xx = fmaxf(xx, g1.x); xy = fmaxf(xy, g1.y); xz = fmaxf(xz, g1.z);
        const int ndl = is_left ? dl : gd, ndr = is_left ? gd : dr;
        const int P = (L == 0 && R == n - 1) ? 0 : (ndr > ndl ? R : L);
        w0 = lo0;
        w1 = make_float4(lo1.x, lo1.y, lo1.z, __int_as_float(2));
        w2 = hi0;
        w3 = make_float4(hi1.x, hi1.y, hi1.z, __int_as_float(0));
        wP = P;
        wl = __float_as_int(lo0.w);
        wr = __float_as_int(hi0.w);
        have = true;
        l = L; r = R; ref = P; dl = ndl; dr = ndr;
    }
    flush();
    return done;
}

template <class Segs, int LANES = kTopLanes>
__global__ void __launch_bounds__(256) k_emit_top(Segs segs, const OpenItem *__restrict__ items, int cap,
                                                  const uint32_t *__restrict__ counts,
                                                  float4 *nodes_all, int32_t *parents_all,
                                                  uint32_t *arrive_all, float4 *pend_all,
                                                  uint8_t *pend_d_all,
                                                  const uint32_t *__restrict__ epoch_p,
                                                  Control *ctl) {
    const int gw = (blockIdx.x * 256 + threadIdx.x) / LANES, lane = threadIdx.x % LANES;
    if (gw >= segs.blocks()) return;
    if (ld_relaxed_gpu(&ctl->err) & ERR_LOOKBACK_TIMEOUT) return;  // unsorted keys: nothing to build
    const int cnt = (int)min(counts[gw], (uint32_t)cap);
    if (lane >= cnt) return;
    const uint32_t epoch = *epoch_p;
    const Span sp = segs.span(gw);
    for (int q = lane; q < cnt; q += LANES)
        if (!top_climb(items[segs.item_base(gw, cap) + q], sp.n, nodes_all + 4ull * sp.start,
                       parents_all + 2ull * sp.start, arrive_all + sp.start, pend_all + 2ull * sp.start,
                       pend_d_all + sp.start, epoch))
            atomicOr(&ctl->err, ERR_CLIMB);
}

// K3c, first level: one block per group of Groups::kBlocks consecutive K3b blocks
// climbs the group's open items through every split both of whose sides lie in the group, in
// shared memory - the same park / merge handshake as K3b, splits found through a hash table,
// each item climbing on its own thread with no barrier between levels - and writes those
// records and parent links.  What is left (items whose next split leaves the group, children
// parked at a split whose sibling never came; about 1 / kBlocks of the items) then climbs on in
// the same block with the arrival words of k_emit_top (top_climb), while other groups still run
// their shared-memory climbs: those touch only splits inside their own groups, the arrival words
// only splits that straddle a group.  (As a kernel of its own after the group pass the global
// climb took 80 us of the 16.7 M build's 155; in the group kernel the pass takes 151 us: the
// chain of arrivals up to the root, not the launch, sets its length.)  A plain build's groups
// span 4096 leaves (16 blocks of 256, or 32 of 128), a batched build's 16 blocks of its meshes.
// A group with more than kGroupCap items climbs them all with the arrival words.
constexpr int kGroupBlocks = 16;  // a batched build's blocks per group
constexpr int kMaxGroupBlocks = 32;
constexpr int kGroupCap = 256;
constexpr int kGroupHash = 512;   // slots (power of two); distinct splits <= 2 x items
constexpr int kGroupThreads = 128;

struct GroupSmem {
    OpenItem it[kGroupCap];
    int out[kGroupCap];
    int hkey[kGroupHash];
    uint32_t hmask[kGroupHash];
    int hidx[kGroupHash][2];
    int bstart[kMaxGroupBlocks + 1];
    int cnt[1];
    int nout;
};

// Where group g lies: its segment (first triangle, size), its tree blocks [blk0, blk1) as
// global block numbers and its first leaf within the segment.  A group never crosses a segment.
struct GroupSpan {
    size_t start;
    int n, blk0, blk1, leaf0;
};
template <int LOG>
struct OneSegGroups {  // plain build: blocks kBlocks g .. kBlocks g + kBlocks - 1 of the one segment
    static constexpr int kBlocks = 4096 >> LOG;
    static_assert(kBlocks <= kMaxGroupBlocks, "one warp scans a group's blocks");
    int n;
    __device__ __forceinline__ GroupSpan group(int g) const {
        const int nblk = (n + (1 << LOG) - 1) >> LOG, b0 = g * kBlocks;
        return GroupSpan{0, n, b0, min(nblk, b0 + kBlocks), b0 << LOG};
    }
};
template <int LOG>
struct ManySegGroups {  // batched build: a segment's blocks in groups of 16, from its first group
    static constexpr int kBlocks = kGroupBlocks;
    const SegRow *rows;
    const uint32_t *grp_seg;
    __device__ __forceinline__ GroupSpan group(int g) const {
        const uint32_t sg = __ldg(grp_seg + g);
        const uint32_t t0 = __ldg(&rows[sg].tri), t1 = __ldg(&rows[sg + 1].tri);
        const int first = (int)__ldg(&rows[sg].blk), end = (int)__ldg(&rows[sg + 1].blk);
        const int b0 = first + (g - (int)__ldg(&rows[sg].grp)) * kGroupBlocks;
        return GroupSpan{t0, (int)(t1 - t0), b0, min(end, b0 + kGroupBlocks), (b0 - first) << LOG};
    }
};

template <int LOG, class Groups>
__global__ void __launch_bounds__(kGroupThreads) k_top_group(Groups groups, const OpenItem *__restrict__ items,
                                                   const uint32_t *__restrict__ counts, float4 *nodes_all,
                                                   int32_t *parents_all, uint32_t *arrive_all, float4 *pend_all,
                                                   uint8_t *pend_d_all, const uint32_t *__restrict__ epoch_p,
                                                   Control *ctl) {
    constexpr int EB = 1 << LOG, GB = Groups::kBlocks;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GroupSmem &S = *reinterpret_cast<GroupSmem *>(smem_raw);
    const int t = threadIdx.x;
    const int g = blockIdx.x;
    chain_wait();
    if (ld_relaxed_gpu(&ctl->err) & ERR_LOOKBACK_TIMEOUT) return;  // unsorted keys: nothing to build
    const GroupSpan gs = groups.group(g);
    const int n = gs.n, blk0 = gs.blk0, blk1 = gs.blk1;
    const int lo_leaf = gs.leaf0, hi_leaf = min(n, gs.leaf0 + (blk1 - blk0) * EB);
    float4 *nodes = nodes_all + 4ull * gs.start;
    int32_t *parents = parents_all + 2ull * gs.start;
    uint32_t *arrive = arrive_all + gs.start;
    float4 *pend = pend_all + 2ull * gs.start;
    uint8_t *pend_d = pend_d_all + gs.start;
    const uint32_t epoch = *epoch_p;
    if (t < 32) {  // the blocks' item counts and their exclusive prefix (one warp)
        const int c = (t < GB && blk0 + t < blk1) ? (int)min(counts[blk0 + t], (uint32_t)kOpenCap) : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (t >= o) incl += y;
        }
        if (t < GB) S.bstart[t] = incl - c;
        if (t == 31) {
            S.bstart[GB] = incl;  // lanes from GB on count zero
            S.cnt[0] = min(incl, kGroupCap);
            S.nout = 0;
        }
    }
    for (int h = t; h < kGroupHash; h += kGroupThreads) {
        S.hkey[h] = -1;
        S.hmask[h] = 0u;
    }
    __syncthreads();
    const int total = S.bstart[GB];  // blocks past blk1 count zero
    if (total > kGroupCap) {
        // more items than shared memory holds: every item climbs with the arrival words
        for (int b = blk0; b < blk1; ++b) {
            const int c = S.bstart[b - blk0 + 1] - S.bstart[b - blk0];
            for (int k = t; k < c; k += kGroupThreads)
                if (!top_climb(items[(size_t)b * kOpenCap + k], n, nodes, parents, arrive, pend, pend_d, epoch))
                    atomicOr(&ctl->err, ERR_CLIMB);
        }
        return;
    }
    // The group's items into shared memory: item `at` of the group is item at - bstart[b] of
    // block blk0 + b.  Each thread holds at most two, and issues both loads before storing
    // either (a loop over the blocks waited for one load per block in turn).
    static_assert(kGroupCap <= 2 * kGroupThreads, "at most two items per thread");
    auto src = [&](int at) -> const OpenItem & {
        int b = 0;
        while (S.bstart[b + 1] <= at) ++b;  // bstart[GB] = total > at: ends at a non-empty block
        return items[(size_t)(blk0 + b) * kOpenCap + (at - S.bstart[b])];
    };
    {
        const int a0 = t, a1 = t + kGroupThreads;
        OpenItem i0, i1;
        if (a0 < total) i0 = src(a0);
        if (a1 < total) i1 = src(a1);
        if (a0 < total) S.it[a0] = i0;
        if (a1 < total) S.it[a1] = i1;
    }
    auto push_out = [&](int i) {
        const int at = atomicAdd(&S.nout, 1);
        S.out[at] = i;  // at most one entry per item: < kGroupCap
    };
    __syncthreads();
    // Every item climbs on its own thread, with no barrier between levels: S.it[i] holds item
    // i's current node; at a split the first child parks (its row and index published by the
    // release of the arrival mask), the second merges both and climbs on with the parent.
    const int count = S.cnt[0];
    for (int i = t; i < count; i += kGroupThreads) {
        OpenItem it = S.it[i];
        for (int step = 0; step < 4 * EB; ++step) {
            const int l = it.xl, r = it.xr, dl = it.pad0, dr = __float_as_int(it.hi.w);
            const bool is_left = dr > dl;
            const int s = is_left ? r : l - 1;
            if (s < lo_leaf || s + 1 >= hi_leaf || s < 0 || s >= n - 1) {
                push_out(i);
                break;
            }
            uint32_t h = ((uint32_t)s * 2654435761u) & (kGroupHash - 1);
            for (int probe = 0; probe < kGroupHash; ++probe) {
                const int prev = atomicCAS(&S.hkey[h], -1, s);
                if (prev == -1 || prev == s) break;
                h = (h + 1) & (kGroupHash - 1);
            }
            const int side = is_left ? 0 : 1;
            S.hidx[h][side] = i;
            if (atom_or_acq_rel_cta(&S.hmask[h], 1u << side) == 0u) break;  // first parks
            const int j = S.hidx[h][side ^ 1];
            const OpenItem sb = S.it[j];
            const int L = is_left ? l : sb.xl, R = is_left ? sb.xr : r;
            const int ndl = is_left ? dl : sb.pad0, ndr = is_left ? __float_as_int(sb.hi.w) : dr;
            const bool root = L == 0 && R == n - 1;
            const int P = root ? 0 : (ndr > ndl ? R : L);
            const OpenItem &lc = is_left ? it : sb;
            const OpenItem &rc = is_left ? sb : it;
            float4 *rec = nodes + 4ull * P;
            rec[0] = lc.lo;
            rec[1] = make_float4(lc.hi.x, lc.hi.y, lc.hi.z, __int_as_float(2));
            rec[2] = rc.lo;
            rec[3] = make_float4(rc.hi.x, rc.hi.y, rc.hi.z, __int_as_float(0));
            const int lref = __float_as_int(lc.lo.w), rref = __float_as_int(rc.lo.w);
            parents[lref >= 0 ? lref : n - (lref + 1)] = P;
            parents[rref >= 0 ? rref : n - (rref + 1)] = P;
            if (root) break;
            OpenItem pa;
            pa.lo = make_float4(fminf(it.lo.x, sb.lo.x), fminf(it.lo.y, sb.lo.y), fminf(it.lo.z, sb.lo.z),
                                __int_as_float(P));
            pa.hi = make_float4(fmaxf(it.hi.x, sb.hi.x), fmaxf(it.hi.y, sb.hi.y), fmaxf(it.hi.z, sb.hi.z),
                                __int_as_float(ndr));
            pa.xl = L;
            pa.xr = R;
            pa.pad0 = ndl;
            pa.pad1 = 0;
            S.it[i] = pa;
            it = pa;
        }
    }
    __syncthreads();
    // a child parked at a split whose sibling never came: its parent leaves the group
    for (int h = t; h < kGroupHash; h += kGroupThreads) {
        const uint32_t mk = S.hmask[h];
        if (mk == 1u || mk == 2u) push_out(S.hidx[h][mk == 1u ? 0 : 1]);
    }
    __syncthreads();
    // what leaves the group climbs on at once with the arrival words, beside the other groups'
    // shared-memory climbs (those touch only splits inside their groups)
    const int nout = S.nout;
    for (int k = t; k < nout; k += kGroupThreads)
        if (!top_climb(S.it[S.out[k]], n, nodes, parents, arrive, pend, pend_d, epoch)) atomicOr(&ctl->err, ERR_CLIMB);
}

// the layout plus the slack that puts it on a 128-byte boundary
template <int LOG, class Segs, class Leaves>
inline size_t leaves_smem_bytes() { return sizeof(typename TreeLayout<LOG, Segs, Leaves>::Smem) + 128; }

// The soup as a 2-D tensor of `rows` rows of 12 floats, 48 bytes apart, for the tree pass's
// tile::gather4 copies: one-row boxes of a whole row, the L2 filling 64 bytes per DRAM request
// (most of a randomly gathered row's 128-byte line is never used).  The base is 16-byte
// aligned (every entry point checks it) and 1 <= rows <= LVBH_MAX_TRIS.
cudaError_t soup_tensor_map(CUtensorMap *m, const float4 *tri, uint32_t rows) {
    static const PFN_cuTensorMapEncodeTiled_v12000 enc = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            f = nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    if (!enc) return cudaErrorNotSupported;
    const cuuint64_t dims[2] = {12, rows}, strides[1] = {48};
    const cuuint32_t box[2] = {12, 1}, elem[2] = {1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float4 *>(tri), dims, strides, box, elem,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_64B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int LOG, class Segs, class Leaves>
void launch_emit_impl(Segs segs, int groups, Leaves lv, const CUtensorMap &soup_map, const uint32_t *keys,
                      float4 *nodes, int32_t *parents,
                      OpenItem *items, uint32_t *counts, uint32_t *arrive, float4 *pend,
                      uint8_t *pend_d, const uint32_t *epoch, Control *ctl, bool top,
                      cudaStream_t s, cudaEvent_t *ev, int ctas_per_sm,
                      const uint32_t *grp_seg = nullptr, int ngroups = 0) {
    if (ev) cudaEventRecord(ev[0], s);  // the leaf gather runs inside the tree pass
    const int per_sm = ctas_per_sm > 0 && ctas_per_sm < TreeGeo<LOG>::kCtasPerSm ? ctas_per_sm
                                                                                : TreeGeo<LOG>::kCtasPerSm;
    const int grid = min(groups, sm_count() * per_sm);
    // batched builds always chain; a one-mesh build by its size
    bool chain = true;
    if constexpr (std::is_same<Segs, OneSeg<LOG>>::value) chain = chain_build((uint32_t)segs.n);
    launch_chained(chain, k_tree_climb<LOG, Segs, Leaves>, grid, TreeGeo<LOG>::EB, leaves_smem_bytes<LOG, Segs, Leaves>(), s,
                   segs, keys, lv, nodes, parents, items, counts, ctl, soup_map);
    if (ev) cudaEventRecord(ev[1], s);
    if (top) {
        if constexpr (std::is_same<Segs, OneSeg<LOG>>::value) {
            constexpr int GB = OneSegGroups<LOG>::kBlocks;
            const int ngroups = (groups + GB - 1) / GB;
            launch_chained(chain, k_top_group<LOG, OneSegGroups<LOG>>, ngroups, kGroupThreads, sizeof(GroupSmem), s,
                           OneSegGroups<LOG>{segs.n}, items, counts, nodes, parents, arrive, pend, pend_d, epoch, ctl);
        } else if (grp_seg) {
            // batched: the same over groups of 16 blocks that never cross a mesh
            const ManySegGroups<LOG> gr{segs.rows, grp_seg};
            if (ngroups > 0)
                launch_chained(chain, k_top_group<LOG, ManySegGroups<LOG>>, ngroups, kGroupThreads, sizeof(GroupSmem), s, gr,
                               items, counts, nodes, parents, arrive, pend, pend_d, epoch, ctl);
        } else {
            k_emit_top<<<(groups * kTopLanes + 255) / 256, 256, 0, s>>>(segs, items, kOpenCap, counts, nodes,
                                                                         parents, arrive, pend, pend_d,
                                                                         epoch, ctl);
        }
    }
    if (ev) cudaEventRecord(ev[2], s);
}

template <class K>
cudaError_t prefer_shared(K kernel, size_t bytes) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared);
}

}  // namespace

size_t emit_groups(uint32_t n, int log_eb) { return (n + (1u << log_eb) - 1) >> log_eb; }

cudaError_t emit_init() {
    constexpr int L = kLogEmitBlock;
    cudaError_t e = prefer_shared(k_tree_climb<L, OneSeg<L>>, leaves_smem_bytes<L, OneSeg<L>, SoupLeaves>());
    if (e == cudaSuccess) e = prefer_shared(k_tree_climb<8, ManySegs<8>>, leaves_smem_bytes<8, ManySegs<8>, SoupLeaves>());
    if (e == cudaSuccess) e = prefer_shared(k_tree_climb<7, ManySegs<7>>, leaves_smem_bytes<7, ManySegs<7>, SoupLeaves>());
    if (e == cudaSuccess)
        e = prefer_shared(k_tree_climb<L, OneSeg<L>, MeshLeaves>, leaves_smem_bytes<L, OneSeg<L>, MeshLeaves>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_top_group<kLogEmitBlock, OneSegGroups<kLogEmitBlock>>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GroupSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_top_group<8, ManySegGroups<8>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(GroupSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_top_group<7, ManySegGroups<7>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(GroupSmem));
    return e;
}

cudaError_t launch_emit(const float4 *tri, const uint32_t *perm, const uint32_t *keys, uint32_t n,
                        float4 *otri, float4 *nodes, int32_t *parents, OpenItem *items,
                        uint32_t *counts, uint32_t *arrive, float4 *pend, uint8_t *pend_d,
                        const uint32_t *epoch, Control *ctl, cudaStream_t s, cudaEvent_t *ev) {
    if (n == 0) return cudaSuccess;
    CUtensorMap map;
    const cudaError_t e = soup_tensor_map(&map, tri, n);
    if (e != cudaSuccess) return e;
    const int groups = (int)emit_groups(n, kLogEmitBlock);
    launch_emit_impl<kLogEmitBlock>(OneSeg<kLogEmitBlock>{(int)n}, groups, SoupLeaves{tri, perm, otri}, map, keys,
                                    nodes, parents, items, counts, arrive, pend, pend_d, epoch,
                                    ctl, groups > 1, s, ev, 0);
    return cudaSuccess;
}

void launch_emit_mesh(const float4 *verts, uint32_t num_verts, const uint32_t *sidx, const uint32_t *keys,
                      uint32_t n, float4 *nodes, int32_t *parents, OpenItem *items, uint32_t *counts,
                      uint32_t *arrive, float4 *pend, uint8_t *pend_d, const uint32_t *epoch, Control *ctl,
                      cudaStream_t s, cudaEvent_t *ev) {
    if (n == 0) return;
    const int groups = (int)emit_groups(n, kLogEmitBlock);
    CUtensorMap unused;  // mesh leaves come by cp.async
    std::memset(&unused, 0, sizeof unused);
    launch_emit_impl<kLogEmitBlock>(OneSeg<kLogEmitBlock>{(int)n}, groups, MeshLeaves{verts, sidx, num_verts},
                                    unused, keys, nodes, parents, items, counts, arrive, pend, pend_d, epoch, ctl,
                                    groups > 1, s, ev, 0);
}

cudaError_t launch_emit_batch(const BatchPlan &bp, const float4 *tri, const uint32_t *perm,
                              const uint32_t *keys, float4 *otri, float4 *nodes, int32_t *parents,
                              OpenItem *items, uint32_t *counts, uint32_t *arrive, float4 *pend,
                              uint8_t *pend_d, const uint32_t *epoch, Control *ctl, cudaStream_t s,
                              cudaEvent_t *ev) {
    if (bp.blocks == 0) return cudaSuccess;
    CUtensorMap map;
    const cudaError_t e = soup_tensor_map(&map, tri, bp.total);
    if (e != cudaSuccess) return e;
    if (bp.log_block == 7)
        launch_emit_impl<7>(ManySegs<7>{bp.rows, bp.blk_seg, (int)bp.blocks}, (int)bp.blocks,
                            SoupLeaves{tri, perm, otri}, map, keys, nodes, parents, items, counts, arrive, pend,
                            pend_d, epoch, ctl, true, s, ev, bp.tree_ctas_per_sm, bp.grp_seg, (int)bp.groups);
    else
        launch_emit_impl<8>(ManySegs<8>{bp.rows, bp.blk_seg, (int)bp.blocks}, (int)bp.blocks,
                            SoupLeaves{tri, perm, otri}, map, keys, nodes, parents, items, counts, arrive, pend,
                            pend_d, epoch, ctl, true, s, ev, bp.tree_ctas_per_sm, bp.grp_seg, (int)bp.groups);
    return cudaSuccess;
}

}  // namespace lvbh
