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
// s with a smaller d.  That node is the LEFT child of split R when d[R] > d[L-1], else the
// RIGHT child of split L-1 (the two values always differ), so its Karras index is R or L (0
// for the root) - exactly the numbering compute_child_index produces.  Its children are the
// nodes with Karras indices s and s+1 (leaves s, s+1 when L == s, R == s+1).  So every node's
// record follows from nearest-smaller-value queries on d alone: no per-node binary search,
// no climbing, no atomics.
//
// Passes.
//   K3a (k_leaf_gather)  one thread per sorted leaf k: gathers triangle perm[k] (3 x 16-byte
//                        loads), writes it to the output soup at k, and writes its box (exact-
//                        zero components nudged by 1e-8 as bvh-up-pass.js:209-210 does) to a
//                        24-byte scratch record.  Random-access bound.
//   K3b (k_tree_leaves)  blocks of 256 sorted leaves, one thread per leaf / split, a persistent
//                        grid that prefetches the next block.  Two sparse tables in shared
//                        memory - minima of d, unions of leaf boxes - give every split its
//                        nearest smaller separators by binary lifting and its children's boxes
//                        by two O(1) range queries, so every node whose range stays inside the
//                        block is completed at once (record and parent links staged in shared
//                        memory and written coalesced).  A node or leaf whose parent split is
//                        not inside the block leaves it as an "open item" (at most 2 x 64 per
//                        block: they hang off the two boundary paths of a tree at most 64 deep).
//   K3c (k_emit_top)     the nodes that straddle blocks (~3 % of them), built bottom-up from
//                        the open items with arrival words (see below).
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

constexpr int EB = kEmitBlock;                 // level 1: leaves (threads) per CTA
constexpr int kLogEB = 8;                      // EB == 1 << kLogEB
constexpr int kTreeCtasPerSm = 3;             // resident K3b CTAs per SM (persistent grid)
constexpr int kTopLanes = 8;                   // K3c threads per block of K3b

__device__ __forceinline__ int dd_global(const uint32_t *__restrict__ keys, int n, int x) {
    if (x < 0 || x >= n - 1) return -1;
    const uint32_t a = __ldg(keys + x), b = __ldg(keys + x + 1);
    return a != b ? __clz(a ^ b) : 32 + __clz(x ^ (x + 1));
}

// Block-wide exclusive sum of one value per thread; returns the thread's offset, *total the sum.
template <int kThreads>
__device__ __forceinline__ int block_excl_sum(int v, int *s_warp, int *total) {
    constexpr int W = kThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    int off = 0, all = 0;
#pragma unroll
    for (int i = 0; i < W; ++i) {
        off += i < warp ? s_warp[i] : 0;
        all += s_warp[i];
    }
    __syncthreads();
    *total = all;
    return off + incl - v;
}

// Where a block of EB sorted leaves lives.  A batched build is a list of segments (meshes)
// laid end to end; every block lies inside one segment and every index a kernel works with
// is local to that segment (the plain build is the one-segment case).
struct Span {
    size_t start;  // the segment's first position in the batch
    int n;         // the segment's triangle count
    int b0;        // the block's first leaf within the segment
};

struct OneSeg {
    int n;
    __device__ __forceinline__ int blocks() const { return (n + EB - 1) / EB; }
    __device__ __forceinline__ Span span(int blk) const { return Span{0, n, blk * EB}; }
};

struct ManySegs {
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
};

// K3a: leaf gather.  One thread per sorted position k: triangle perm[k] (3 x 16-byte loads)
// to the output soup at k, its box (exact-zero components nudged by 1e-8 as
// bvh-up-pass.js:209-210 does) to lbox[k] (min xyz, max xyz: 24 bytes).
template <class Segs>
__global__ void __launch_bounds__(256) k_leaf_gather(Segs segs, const float4 *__restrict__ tri,
                                                     const uint32_t *__restrict__ perm,
                                                     float4 *__restrict__ otri,
                                                     float2 *__restrict__ lbox, Control *ctl) {
    const Span sp = segs.span(blockIdx.x);
    const int kl = sp.b0 + threadIdx.x;
    if (kl >= sp.n) return;
    const size_t k = sp.start + kl;
    uint32_t ti = __ldg(perm + k);
    if (ti >= (uint32_t)sp.n) { atomicOr(&ctl->err, ERR_CLIMB); ti = 0; }
    const float4 *src = tri + 3ull * (sp.start + ti);
    const float4 a = __ldg(src), b = __ldg(src + 1), c = __ldg(src + 2);
    st_stream(otri + 3ull * k, a);
    st_stream(otri + 3ull * k + 1, b);
    st_stream(otri + 3ull * k + 2, c);
    float nx = fminf(a.x, fminf(b.x, c.x)), ny = fminf(a.y, fminf(b.y, c.y)), nz = fminf(a.z, fminf(b.z, c.z));
    float xx = fmaxf(a.x, fmaxf(b.x, c.x)), xy = fmaxf(a.y, fmaxf(b.y, c.y)), xz = fmaxf(a.z, fmaxf(b.z, c.z));
    nx = nx == 0.0f ? -1e-8f : nx; ny = ny == 0.0f ? -1e-8f : ny; nz = nz == 0.0f ? -1e-8f : nz;
    xx = xx == 0.0f ? 1e-8f : xx;  xy = xy == 0.0f ? 1e-8f : xy;  xz = xz == 0.0f ? 1e-8f : xz;
    lbox[3ull * k] = make_float2(nx, ny);
    lbox[3ull * k + 1] = make_float2(nz, xx);
    lbox[3ull * k + 2] = make_float2(xy, xz);
}

// K3b shared memory: sparse tables over one block of EB leaves.
//   md[l][x] = min of S[x .. x + 2^l - 1] (S[x] = d[b0 + x - 1], x in [0, EB])
//   bx[l][c][x] = component c (min xyz, max xyz) of the union of leaf boxes x .. x + 2^l - 1
// The records of the block are staged over bx once the range queries are done.
struct LeafTables {
    int8_t md[kLogEB + 1][EB + 4];
    union {
        float bx[kLogEB + 1][6][EB];
        float4 rec[EB][4];  // records of the nodes completed here, by index - b0
    };
    int pint[EB];        // parent of internal node b0 + j (-1 = not set here)
    int pleaf[EB];       // parent of leaf b0 + j (-1 = not set here)
    uint32_t key[EB + 2];
    uint8_t recv[EB];
    uint8_t local[EB];   // split b0 + j stays inside the block
    uint8_t open[EB];    // an open item starts at leaf b0 + j
    int16_t pos[EB];     // its position among the block's open items
    int warp[EB / 32];
};

// Union of leaf boxes [a, b] (0 <= a <= b < EB) from the box table.
__device__ __forceinline__ void range_box(const LeafTables &T, int a, int b, float4 &lo, float4 &hi) {
    const int l = 31 - __clz(b - a + 1);
    const int c = b - (1 << l) + 1;
    lo = make_float4(fminf(T.bx[l][0][a], T.bx[l][0][c]), fminf(T.bx[l][1][a], T.bx[l][1][c]),
                     fminf(T.bx[l][2][a], T.bx[l][2][c]), 0.f);
    hi = make_float4(fmaxf(T.bx[l][3][a], T.bx[l][3][c]), fmaxf(T.bx[l][4][a], T.bx[l][4][c]),
                     fmaxf(T.bx[l][5][a], T.bx[l][5][c]), 0.f);
}

// K3b: the tree over blocks of EB sorted leaves; a persistent grid walks the blocks and
// fetches the next block's keys and leaf boxes while it works on the current one.  Every
// split whose node stays inside the block finds its node range by binary lifting on the d
// table (nearest smaller separators on both sides), its Karras index and children from that
// range, and its children's boxes by two range queries on the box table: all nodes of a block
// complete at once.  The nodes that straddle blocks are left to K3c as open items.
template <class Segs>
__global__ void __launch_bounds__(EB) k_tree_leaves(Segs segs, const uint32_t *__restrict__ keys_all,
                                                    const float2 *__restrict__ lbox_all,
                                                    float4 *nodes_all, int32_t *parents_all,
                                                    OpenItem *out_items, uint32_t *out_counts,
                                                    Control *ctl) {
    extern __shared__ __align__(16) unsigned char smem[];
    LeafTables &T = *reinterpret_cast<LeafTables *>(smem);
    const int t = threadIdx.x;
    const int nblk = segs.blocks();

    // registers of the next block: its span, this thread's key and leaf box, the two edge keys
    Span nsp{0, 0, 0};
    uint32_t nk = 0, nk_lo = 0, nk_hi = 0;
    float2 np0 = make_float2(0.f, 0.f), np1 = np0, np2 = np0;
    auto fetch = [&](int blk) {
        nsp = segs.span(blk);
        const uint32_t *keys = keys_all + nsp.start;
        const float2 *lbox = lbox_all + 3ull * nsp.start;
        const int b0 = nsp.b0, n = nsp.n, k = b0 + t;
        if (k < n) {
            nk = __ldg(keys + k);
            np0 = __ldg(lbox + 3ull * k); np1 = __ldg(lbox + 3ull * k + 1); np2 = __ldg(lbox + 3ull * k + 2);
        }
        if (t == 0) nk_lo = b0 > 0 ? __ldg(keys + b0 - 1) : 0u;
        if (t == EB - 1) nk_hi = (b0 + EB < n) ? __ldg(keys + b0 + EB) : 0u;
    };
    if ((int)blockIdx.x < nblk) fetch(blockIdx.x);

    for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const Span sp = nsp;
        const int b0 = sp.b0, n = sp.n;
        float4 *nodes = nodes_all + 4ull * sp.start;
        int32_t *parents = parents_all + 2ull * sp.start;
        const int m = min(EB, n - b0);
        const int k = b0 + t;
        const bool active = t < m;
        T.key[t + 1] = active ? nk : 0u;
        if (t == 0) T.key[0] = nk_lo;
        if (t == EB - 1) T.key[EB + 1] = nk_hi;
        const float box[6] = {np0.x, np0.y, np1.x, np1.y, np2.x, np2.y};
#pragma unroll
        for (int c = 0; c < 6; ++c) T.bx[0][c][t] = active ? box[c] : 0.f;
        T.pint[t] = -1;
        T.pleaf[t] = -1;
        T.recv[t] = 0;
        T.open[t] = 0;
        T.local[t] = 0;
        if (blk + (int)gridDim.x < nblk) fetch(blk + gridDim.x);
        if (n == 1) {  // one leaf, one arrival at node 0: left slot only, f_1 = 1
            if (t == 0) {
                nodes[0] = make_float4(box[0], box[1], box[2], __int_as_float(-1));
                nodes[1] = make_float4(box[3], box[4], box[5], __int_as_float(1));
                nodes[2] = make_float4(0.f, 0.f, 0.f, 0.f);
                nodes[3] = make_float4(0.f, 0.f, 0.f, 0.f);
                parents[0] = 0;
                parents[1] = 0;
                out_counts[blk] = 0;
            }
            continue;  // uniform across the block; the tables are untouched by other threads
        }
        if (k == 0) {  // the root has no parent; slot N-1 and record N-1 stay zero
            parents[0] = 0;
            parents[n - 1] = 0;
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            float4 *last = nodes + 4ull * (n - 1);
            last[0] = z; last[1] = z; last[2] = z; last[3] = z;
        }
        __syncthreads();
        auto window_d = [&](int x) -> int {  // x in [b0-1, b0+EB-1]
            if (x < 0 || x >= n - 1) return -1;
            const uint32_t a = T.key[x - b0 + 1], b = T.key[x - b0 + 2];
            return a != b ? __clz(a ^ b) : 32 + __clz(x ^ (x + 1));
        };
        T.md[0][t] = (int8_t)window_d(b0 - 1 + t);
        if (t == 0) T.md[0][EB] = (int8_t)window_d(b0 + EB - 1);
        __syncthreads();
        // sparse tables
#pragma unroll 1
        for (int l = 1; l <= kLogEB; ++l) {
            const int h = 1 << (l - 1);
            if (t + (1 << l) - 1 <= EB) T.md[l][t] = min(T.md[l - 1][t], T.md[l - 1][t + h]);
            if (t + (1 << l) - 1 < m) {
#pragma unroll
                for (int c = 0; c < 3; ++c) T.bx[l][c][t] = fminf(T.bx[l - 1][c][t], T.bx[l - 1][c][t + h]);
#pragma unroll
                for (int c = 3; c < 6; ++c) T.bx[l][c][t] = fmaxf(T.bx[l - 1][c][t], T.bx[l - 1][c][t + h]);
            }
            __syncthreads();
        }

        // split j = t (between leaves b0 + j and b0 + j + 1), its separator S[q], q = j + 1
        const int j = t, q = t + 1;
        int il = -1, ir = -1;
        if (j < m - 1) {
            const int v = T.md[0][q];
            int pos = q;
#pragma unroll
            for (int l = kLogEB; l >= 0; --l)
                if (pos - (1 << l) >= 0 && T.md[l][pos - (1 << l)] >= v) pos -= 1 << l;
            const int a = pos - 1;  // nearest smaller on the left, or -1
            pos = q;
#pragma unroll
            for (int l = kLogEB; l >= 0; --l)
                if (pos + (1 << l) <= m && T.md[l][pos + 1] >= v) pos += 1 << l;
            const int b = pos + 1;  // nearest smaller on the right, or past the window
            if (a >= 0 && b <= m) {
                il = a;
                ir = b - 1;
                T.local[j] = 1;
            }
        }
        __syncthreads();

        auto S = [&](int x) -> int { return T.md[0][x]; };
        auto split_local = [&](int ps) -> bool { return ps >= 0 && ps < m - 1 && T.local[ps]; };
        int P = 0;
        bool node_open = false;
        float4 w0, w1, w2, w3;
        if (il >= 0) {
            const bool root = (b0 + il == 0) && (b0 + ir == n - 1);
            const bool left_child = S(ir + 1) > S(il);
            P = root ? 0 : (left_child ? b0 + ir : b0 + il);
            const int lref = (il == j) ? -(b0 + j + 1) : b0 + j;
            const int rref = (ir == j + 1) ? -(b0 + j + 2) : b0 + j + 1;
            float4 l0, l1, r0, r1;
            range_box(T, il, j, l0, l1);
            range_box(T, j + 1, ir, r0, r1);
            w0 = make_float4(l0.x, l0.y, l0.z, __int_as_float(lref));
            w1 = make_float4(l1.x, l1.y, l1.z, __int_as_float(2));
            w2 = make_float4(r0.x, r0.y, r0.z, __int_as_float(rref));
            w3 = make_float4(r1.x, r1.y, r1.z, __int_as_float(0));
            T.recv[P - b0] = 1;
            if (lref >= 0) T.pint[lref - b0] = P; else T.pleaf[-(lref + 1) - b0] = P;
            if (rref >= 0) T.pint[rref - b0] = P; else T.pleaf[-(rref + 1) - b0] = P;
            node_open = !root && !split_local(left_child ? ir : il - 1);
            if (node_open) T.open[il] = 1;
        }
        bool leaf_open = false;
        if (active) {  // a leaf whose parent split is not local leaves the block as it is
            const int ps = S(t + 1) > S(t) ? t : t - 1;
            leaf_open = !split_local(ps);
            if (leaf_open) T.open[t] = 1;
        }
        __syncthreads();

        // open items in leaf order: the item starting at leaf t takes position pos[t]
        int total;
        const int f = T.open[t];
        T.pos[t] = (int16_t)block_excl_sum<EB>(f, T.warp, &total);
        __syncthreads();
        OpenItem *out = out_items + (size_t)blk * kOpenCap;
        auto emit_open = [&](int a, int b, int ref) {
            const int at = T.pos[a];
            if (at >= kOpenCap) { atomicOr(&ctl->err, ERR_CLIMB); return; }
            float4 lo, hi;
            range_box(T, a, b, lo, hi);
            OpenItem it;
            it.lo = make_float4(lo.x, lo.y, lo.z, __int_as_float(ref));
            it.hi = make_float4(hi.x, hi.y, hi.z, __int_as_float(S(b + 1)));
            it.xl = b0 + a;
            it.xr = b0 + b;
            it.pad0 = it.pad1 = 0;
            out[at] = it;
        };
        if (leaf_open) emit_open(t, t, -(k + 1));
        if (node_open) emit_open(il, ir, P);
        if (t == 0) out_counts[blk] = (uint32_t)min(total, kOpenCap);
        if (t == 0 && total > kOpenCap) atomicOr(&ctl->err, ERR_CLIMB);
        __syncthreads();  // the box table is done with: stage the records over it
        if (il >= 0) {
            float4 *rc = T.rec[P - b0];
            rc[0] = w0; rc[1] = w1; rc[2] = w2; rc[3] = w3;
        }
        __syncthreads();
        // records and parent links, coalesced
        if (active) {
            if (T.recv[t]) {
                float4 *dst = nodes + 4ull * k;
                dst[0] = T.rec[t][0]; dst[1] = T.rec[t][1]; dst[2] = T.rec[t][2]; dst[3] = T.rec[t][3];
            }
            if (T.pint[t] >= 0) parents[k] = T.pint[t];
            if (T.pleaf[t] >= 0) parents[n + k] = T.pleaf[t];
        }
        __syncthreads();  // before the next block overwrites the tables
    }
}

// K3c: the nodes that straddle blocks.  kTopLanes threads per block of K3b; each climbs one of
// the block's open items (a block leaves about 8) through the remaining splits.  At a split the first arriving child parks
// its box, link and far range end in pend[] at its own index (r when it is a left child, l
// when a right child - no two pending children ever share one), fences, and exchanges the
// build's epoch into the split's arrival word; the second, seeing the epoch already there,
// reads its sibling back, merges, finds the parent's range and Karras index and writes the
// record and both parent links.  Nothing waits, so the kernel cannot hang; climbs are bounded
// and every index is range-checked.  The epoch makes the arrival words reusable without
// clearing: a word left by an older build never equals the current epoch.
template <class Segs>
__global__ void __launch_bounds__(256) k_emit_top(Segs segs, const OpenItem *__restrict__ items,
                                                  const uint32_t *__restrict__ counts,
                                                  const uint32_t *__restrict__ keys_all,
                                                  float4 *nodes_all, int32_t *parents_all,
                                                  uint32_t *arrive_all, float4 *pend_all,
                                                  const uint32_t *__restrict__ epoch_p,
                                                  Control *ctl) {
    const int gw = (blockIdx.x * 256 + threadIdx.x) / kTopLanes, lane = threadIdx.x % kTopLanes;
    if (gw >= segs.blocks()) return;
    const int cnt = (int)min(counts[gw], (uint32_t)kOpenCap);
    if (lane >= cnt) return;
    const uint32_t epoch = *epoch_p;
    const Span sp = segs.span(gw);
    const int n = sp.n;
    const uint32_t *keys = keys_all + sp.start;
    float4 *nodes = nodes_all + 4ull * sp.start;
    int32_t *parents = parents_all + 2ull * sp.start;
    uint32_t *arrive = arrive_all + sp.start;
    float4 *pend = pend_all + 2ull * sp.start;
    for (int q = lane; q < cnt; q += kTopLanes) {
        const OpenItem it = items[(size_t)gw * kOpenCap + q];
        int l = it.xl, r = it.xr, ref = __float_as_int(it.lo.w);
        float nx = it.lo.x, ny = it.lo.y, nz = it.lo.z, xx = it.hi.x, xy = it.hi.y, xz = it.hi.z;
        int dl = dd_global(keys, n, l - 1), dr = __float_as_int(it.hi.w);
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
            __threadfence();
            if (atomicExch(arrive + s, epoch) != epoch) { done = true; break; }  // first arrival
            __threadfence();
            const float4 g0 = __ldcg(pend + 2ull * sib), g1 = __ldcg(pend + 2ull * sib + 1);
            const int sib_ref = __float_as_int(g0.w), sib_far = __float_as_int(g1.w);
            const int L = is_left ? l : sib_far, R = is_left ? sib_far : r;
            if (L < 0 || R >= n || L > l || R < r || sib_ref < -n || sib_ref >= n - 1) break;
            const float4 lo0 = is_left ? h0 : g0, lo1 = is_left ? h1 : g1;
            const float4 hi0 = is_left ? g0 : h0, hi1 = is_left ? g1 : h1;
            nx = fminf(nx, g0.x); ny = fminf(ny, g0.y); nz = fminf(nz, g0.z);
            xx = fmaxf(xx, g1.x); xy = fmaxf(xy, g1.y); xz = fmaxf(xz, g1.z);
            const int ndl = dd_global(keys, n, L - 1), ndr = dd_global(keys, n, R);
            const int P = (L == 0 && R == n - 1) ? 0 : (ndr > ndl ? R : L);
            float4 *rc = nodes + 4ull * P;
            rc[0] = lo0;
            rc[1] = make_float4(lo1.x, lo1.y, lo1.z, __int_as_float(2));
            rc[2] = hi0;
            rc[3] = make_float4(hi1.x, hi1.y, hi1.z, __int_as_float(0));
            const int lref = __float_as_int(lo0.w), rref = __float_as_int(hi0.w);
            parents[lref >= 0 ? lref : n - (lref + 1)] = P;
            parents[rref >= 0 ? rref : n - (rref + 1)] = P;
            l = L; r = R; ref = P; dl = ndl; dr = ndr;
        }
        if (!done) atomicOr(&ctl->err, ERR_CLIMB);
    }
}

inline size_t leaves_smem_bytes() { return sizeof(LeafTables); }

template <class Segs>
void launch_emit_impl(Segs segs, int groups, const float4 *tri, const uint32_t *perm,
                      const uint32_t *keys, float4 *otri, float4 *nodes, int32_t *parents,
                      float2 *lbox, OpenItem *items, uint32_t *counts, uint32_t *arrive,
                      float4 *pend, const uint32_t *epoch, Control *ctl, bool top,
                      cudaStream_t s, cudaEvent_t *ev) {
    k_leaf_gather<<<groups, 256, 0, s>>>(segs, tri, perm, otri, lbox, ctl);
    if (ev) cudaEventRecord(ev[0], s);
    const int grid = min(groups, sm_count() * kTreeCtasPerSm);
    k_tree_leaves<<<grid, EB, leaves_smem_bytes(), s>>>(segs, keys, lbox, nodes, parents, items,
                                                         counts, ctl);
    if (ev) cudaEventRecord(ev[1], s);
    if (top)
        k_emit_top<<<(groups * kTopLanes + 255) / 256, 256, 0, s>>>(segs, items, counts, keys, nodes,
                                                                     parents, arrive, pend, epoch,
                                                                     ctl);
    if (ev) cudaEventRecord(ev[2], s);
}

template <class K>
cudaError_t prefer_shared(K kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)leaves_smem_bytes());
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                (int)cudaSharedmemCarveoutMaxShared);
}

}  // namespace

size_t emit_groups(uint32_t n) { return (n + EB - 1) / EB; }

cudaError_t emit_init() {
    cudaError_t e = prefer_shared(k_tree_leaves<OneSeg>);
    if (e != cudaSuccess) return e;
    return prefer_shared(k_tree_leaves<ManySegs>);
}

void launch_emit(const float4 *tri, const uint32_t *perm, const uint32_t *keys, uint32_t n,
                 float4 *otri, float4 *nodes, int32_t *parents, float2 *lbox, OpenItem *items,
                 uint32_t *counts, uint32_t *arrive, float4 *pend, const uint32_t *epoch,
                 Control *ctl, cudaStream_t s, cudaEvent_t *ev) {
    if (n == 0) return;
    const int groups = (int)emit_groups(n);
    launch_emit_impl(OneSeg{(int)n}, groups, tri, perm, keys, otri, nodes, parents, lbox, items,
                     counts, arrive, pend, epoch, ctl, groups > 1, s, ev);
}

void launch_emit_batch(const BatchPlan &bp, const float4 *tri, const uint32_t *perm,
                       const uint32_t *keys, float4 *otri, float4 *nodes, int32_t *parents,
                       float2 *lbox, OpenItem *items, uint32_t *counts, uint32_t *arrive,
                       float4 *pend, const uint32_t *epoch, Control *ctl, cudaStream_t s,
                       cudaEvent_t *ev) {
    if (bp.blocks == 0) return;
    launch_emit_impl(ManySegs{bp.rows, bp.blk_seg, (int)bp.blocks}, (int)bp.blocks, tri, perm, keys,
                     otri, nodes, parents, lbox, items, counts, arrive, pend, epoch, ctl, true, s,
                     ev);
}

}  // namespace lvbh
