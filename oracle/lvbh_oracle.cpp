// lvbh_oracle.cpp - CPU restatement of the reference LBVH build.  TEST INFRASTRUCTURE ONLY.
//
// This file is the parity oracle and the timed CPU baseline.  It is never linked into,
// loaded by or called from the product library: only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline / reference arm use it, as the checker.
//
// It restates, step by step, the WGSL compute shaders of AddisonPrairie/WebGPU-LVBH-demo
// (file:line cited per function) with the semantics WGSL defines for them:
//   * f32 arithmetic is IEEE single precision, each operation rounded, no contraction
//     (built with -ffp-contract=off, no fast-math).  WGSL lets f32 `/` be off by 2.5 ULP;
//     this restatement defines it as correctly rounded division (the builder's contract).
//   * f32 -> u32 conversion truncates toward zero and saturates; NaN converts to 0.
//   * i32 arithmetic wraps; integer division by zero yields the dividend.
//   * min/max on f32 are `a < b ? a : b` / `a > b ? a : b` (inputs are NaN-free).
//
// Parity status: UNPINNED against a run of the reference.  The reference has no tests,
// golden vectors or fixtures, and it cannot run here (browser WebGPU; no node, no graphics
// stack).  This restatement is cross-checked against an independent literal Python
// simulation of the same WGSL (tests/golden/make_golden.py), against std::stable_sort, and
// against hand-derived known answers.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp -shared).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline float fmin_w(float a, float b) { return a < b ? a : b; }
inline float fmax_w(float a, float b) { return a > b ? a : b; }

// WGSL u32(f32): truncate toward zero, clamp to [0, 2^32-1], NaN -> 0.
inline uint32_t f32_to_u32(float x) {
    if (!(x == x)) return 0u;
    if (x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

// split_3 (scripts/bvh/kernels/aabb-z-idx.js:202-209).
inline uint32_t split_3(uint32_t u) {
    uint32_t x = u;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// morton_code (scripts/bvh/kernels/aabb-z-idx.js:197-199).
inline uint32_t morton_code(uint32_t x, uint32_t y, uint32_t z) {
    return split_3(x) | (split_3(y) << 1) | (split_3(z) << 2);
}

// WGSL i32 helpers for the split loop of compute_child_index.
inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
inline int32_t wrap_mul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
inline int32_t wgsl_div(int32_t a, int32_t b) {
    if (b == 0) return a;
    if (a == INT32_MIN && b == -1) return a;
    return a / b;
}

int num_threads(int threads) {
#ifdef _OPENMP
    if (threads <= 0) return omp_get_max_threads();
    return threads;
#else
    (void)threads;
    return 1;
#endif
}

}  // namespace

extern "C" {

// Scene box as parse-obj.js:27-53 computes it on the host: min / max of every vertex
// coordinate (over the f32 values the GPU receives).
void oracle_scene_bounds(const float *tri, uint32_t n, float *bounds6) {
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    if (n == 0) {
        for (int a = 0; a < 3; ++a) { bounds6[a] = mn[a]; bounds6[3 + a] = mx[a]; }
        return;
    }
    for (int a = 0; a < 3; ++a) { mn[a] = tri[a]; mx[a] = tri[a]; }
    for (uint64_t i = 0; i < n; ++i) {
        for (int v = 0; v < 3; ++v) {
            const float *p = tri + 12 * i + 4 * v;
            for (int a = 0; a < 3; ++a) { mn[a] = fmin_w(mn[a], p[a]); mx[a] = fmax_w(mx[a], p[a]); }
        }
    }
    for (int a = 0; a < 3; ++a) { bounds6[a] = mn[a]; bounds6[3 + a] = mx[a]; }
}

// compute_aabb_z_idx (scripts/bvh/kernels/aabb-z-idx.js:177-195).
//   aabb8: 8 floats per triangle {min xyz, pad, max xyz, pad} (the AABB_BUFFER), may be NULL.
//   keys : Morton key per triangle in input order.
void oracle_aabb_zidx(const float *tri, uint32_t n, const float *bounds6, float *aabb8,
                      uint32_t *keys, int threads) {
    const float umin[3] = {bounds6[0], bounds6[1], bounds6[2]};
    const float umax[3] = {bounds6[3], bounds6[4], bounds6[5]};
    const float scale = 1023.99f;
#pragma omp parallel for schedule(static) num_threads(num_threads(threads))
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float *t = tri + 12 * i;
        float bmin[3], bmax[3], q[3];
        for (int a = 0; a < 3; ++a) {
            // box.min = min(v0, min(v1, v2)); box.max = max(v0, max(v1, v2))   (:186-187)
            bmin[a] = fmin_w(t[a], fmin_w(t[4 + a], t[8 + a]));
            bmax[a] = fmax_w(t[a], fmax_w(t[4 + a], t[8 + a]));
            // cen = (box.max + box.min) * .5f                                    (:191)
            float cen = (bmax[a] + bmin[a]) * 0.5f;
            // rel = (cen - min) / (max - min)                                    (:192)
            float rel = (cen - umin[a]) / (umax[a] - umin[a]);
            // vec3u(rel * 1023.99f)                                              (:194)
            q[a] = rel * scale;
        }
        if (aabb8) {
            float *o = aabb8 + 8 * i;
            o[0] = bmin[0]; o[1] = bmin[1]; o[2] = bmin[2]; o[3] = 0.0f;
            o[4] = bmax[0]; o[5] = bmax[1]; o[6] = bmax[2]; o[7] = 0.0f;
        }
        keys[i] = morton_code(f32_to_u32(q[0]), f32_to_u32(q[1]), f32_to_u32(q[2]));
    }
}

// The radix sort of scripts/bvh/kernels/radix-sort.js: a stable LSD counting sort with
// 2-bit digits over 16 passes (:486-488), each pass being
//   init_off      (:539-570)  per-workgroup (256 keys) digit counts -> L1
//   scan_up  x2   (:763-803)  exclusive scans of L1 in blocks of 256, then of the block
//                             totals (L2); the grand totals land in L3
//   scan_and_sort (:575-629)  per-workgroup exclusive scan of per-thread (4 key) counts,
//                             plus the L3 digit base, L1 and L2 offsets -> scatter
// with init_idx (:526-534) first.  Keys are sorted in place; idx receives the permutation.
// The reference caps the hierarchy at 2^24 keys (:189-202); this restatement does not.
void oracle_radix_sort(uint32_t *keys, uint32_t n, int32_t *idx, int threads) {
    if (n == 0) return;
    const int nt = num_threads(threads);
    const uint64_t wg_count = (n + 255u) / 256u;          // ceil(size / 256) (:406,476)
    const uint64_t l2_count = (wg_count + 255u) / 256u;   // ceil(size / 65536) (:429)
    std::vector<uint32_t> vals2(n);
    std::vector<int32_t> idx2(n);
    std::vector<uint32_t> l1(wg_count * 4), l2(l2_count * 4);
    uint32_t *vals_buf[2] = {keys, vals2.data()};
    int32_t *idx_buf[2] = {idx, idx2.data()};

    // init_idx (:526-534)
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t i = 0; i < (int64_t)n; ++i) idx[i] = (int32_t)i;

    for (uint32_t k = 0; k < 16; ++k) {
        const uint32_t *vals = vals_buf[k % 2];
        const int32_t *ids = idx_buf[k % 2];
        uint32_t *n_vals = vals_buf[(k + 1) % 2];
        int32_t *n_ids = idx_buf[(k + 1) % 2];
        const uint32_t sh = 2u * k;

        // init_off: workgroup g of 64 threads x 4 consecutive keys counts its digits.
#pragma omp parallel for schedule(static) num_threads(nt)
        for (int64_t g = 0; g < (int64_t)wg_count; ++g) {
            uint32_t c[4] = {0, 0, 0, 0};
            for (uint64_t e = 256u * g; e < std::min<uint64_t>(256u * (g + 1), n); ++e)
                c[(vals[e] >> sh) & 3u]++;
            for (int d = 0; d < 4; ++d) l1[4 * g + d] = c[d];
        }
        // scan_up level 1: exclusive scan of L1 inside each block of 256 entries; block
        // totals -> L2.
        for (uint64_t b = 0; b < l2_count; ++b) {
            uint32_t run[4] = {0, 0, 0, 0};
            for (uint64_t g = 256u * b; g < std::min<uint64_t>(256u * (b + 1), wg_count); ++g)
                for (int d = 0; d < 4; ++d) { uint32_t c = l1[4 * g + d]; l1[4 * g + d] = run[d]; run[d] += c; }
            for (int d = 0; d < 4; ++d) l2[4 * b + d] = run[d];
        }
        // scan_up level 2: exclusive scan of L2; grand totals -> L3.
        uint32_t l3[4] = {0, 0, 0, 0};
        for (uint64_t b = 0; b < l2_count; ++b)
            for (int d = 0; d < 4; ++d) { uint32_t c = l2[4 * b + d]; l2[4 * b + d] = l3[d]; l3[d] += c; }
        // global_offsets = dot(prefix mask, l3) (:611-614)
        const uint32_t base[4] = {0u, l3[0], l3[0] + l3[1], l3[0] + l3[1] + l3[2]};

        // scan_and_sort: thread t of workgroup g holds keys 256g + 4t + i; its offsets are
        // the workgroup-exclusive scan of per-thread counts plus the running count inside
        // the thread (:592-606), plus the global, L1 and L2 offsets (:611-618).
#pragma omp parallel for schedule(static) num_threads(nt)
        for (int64_t g = 0; g < (int64_t)wg_count; ++g) {
            uint32_t off[4];
            for (int d = 0; d < 4; ++d) off[d] = base[d] + l1[4 * g + d] + l2[4 * (g / 256) + d];
            for (uint64_t e = 256u * g; e < std::min<uint64_t>(256u * (g + 1), n); ++e) {
                uint32_t v = vals[e];
                uint32_t d = (v >> sh) & 3u;
                uint32_t dst = off[d]++;
                n_ids[dst] = ids[e];
                n_vals[dst] = v;
            }
        }
    }
    // 16 passes: the result is back in the caller's buffers (:498-499).
}

// dif / del (scripts/bvh/kernels/radix-tree.js:160-185).
static inline int32_t ref_dif(uint32_t a, uint32_t b) {
    // first differing bit from the MSB, -1 if equal (the loop at :161-168)
    uint32_t x = a ^ b;
    return x == 0 ? -1 : (int32_t)__builtin_clz(x);
}
static inline int32_t ref_del(const uint32_t *keys, int32_t num, int32_t i1, int32_t i2) {
    if (i1 >= num || i2 >= num || i1 < 0 || i2 < 0) return -1;
    int32_t kd = ref_dif(keys[i1], keys[i2]);
    if (kd == -1) kd = 32 + ref_dif((uint32_t)i1, (uint32_t)i2);
    return kd;
}

// compute_radix_tree_pointers + compute_child_index (scripts/bvh/kernels/radix-tree.js:137-238).
// parents: 2N int32, zeroed here (WebGPU buffers start zeroed); root and slot N-1 stay 0.
void oracle_radix_tree(const uint32_t *keys, uint32_t n, int32_t *parents, int threads) {
    if (n == 0) return;
    std::memset(parents, 0, sizeof(int32_t) * 2 * (size_t)n);
    const int32_t num = (int32_t)n;
#pragma omp parallel for schedule(static) num_threads(num_threads(threads))
    for (int64_t ii = 0; ii < (int64_t)num - 1; ++ii) {
        const int32_t i = (int32_t)ii;
        const int32_t dl = ref_del(keys, num, i, i + 1) - ref_del(keys, num, i, i - 1);
        const int32_t d = (dl > 0) - (dl < 0);                 // sign(...)  (:190)
        const int32_t del_min = ref_del(keys, num, i, i - d);  // (:193)
        int32_t l_max = 2;
        while (ref_del(keys, num, i, i + l_max * d) > del_min) l_max *= 2;   // (:195-197)
        int32_t l = 0;
        for (int32_t t = l_max / 2; t > 0; t /= 2)                           // (:200-210)
            if (ref_del(keys, num, i, i + (l + t) * d) > del_min) l += t;
        const int32_t j = i + l * d;
        const int32_t del_node = ref_del(keys, num, i, j);                   // (:213)
        int32_t s = 0;
        {   // (:214-225): t = (l - 1 + v) / v with v doubling in wrapping i32 until t == 0
            int32_t v = 2;
            int32_t t = wgsl_div(wrap_add(l - 1, v), v);
            while (t > 0) {
                if (ref_del(keys, num, i, i + (s + t) * d) > del_node) s += t;
                v = wrap_mul(v, 2);
                t = wgsl_div(wrap_add(l - 1, v), v);
            }
        }
        const int32_t gamma = i + s * d + std::min(d, 0);                    // (:226)
        int32_t px = gamma, py = gamma + 1;
        if (std::min(i, j) == gamma) px = -px - 1;                           // (:229-235)
        if (std::max(i, j) == gamma + 1) py = -py - 1;
        // (:146-156)
        if (px >= 0) parents[px] = i; else parents[num + -(px + 1)] = i;
        if (py >= 0) parents[py] = i; else parents[num + -(py + 1)] = i;
    }
}

// bvh_upward_pass (scripts/bvh/kernels/bvh-up-pass.js:200-280), run as the leaf threads
// 0..N-1 one after another (with threads > 1: concurrently, the left slot published with a
// release flag instead of the reference's 0.0 sentinels, which the same protocol spins on).
// idx: permutation; aabb8: per-triangle boxes in input order; nodes: 16 words per node, N
// nodes, zeroed here.  The output is in arrival order; oracle_canonicalize() sorts it.
void oracle_up_pass(const int32_t *idx, const float *aabb8, const int32_t *parents, uint32_t n,
                    uint32_t *nodes, int threads) {
    if (n == 0) return;
    std::memset(nodes, 0, 64 * (size_t)n);
    const int32_t num = (int32_t)n;
    const int nt = num_threads(threads);
    std::vector<std::atomic<uint32_t>> ready(nt > 1 ? n : 0);
    for (auto &r : ready) r.store(0, std::memory_order_relaxed);
    auto f32 = [](float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; };
    auto u2f = [](uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; };

#pragma omp parallel for schedule(dynamic, 4096) num_threads(nt)
    for (int64_t ii = 0; ii < (int64_t)num; ++ii) {
        const int32_t idx0 = (int32_t)ii;
        const float *bb = aabb8 + 8 * (size_t)idx[idx0];
        float bmin[3] = {bb[0], bb[1], bb[2]}, bmax[3] = {bb[4], bb[5], bb[6]};
        // bbox.min -= (min == 0) * 1e-8f; bbox.max += (max == 0) * 1e-8f   (:209-210)
        for (int a = 0; a < 3; ++a) {
            bmin[a] = bmin[a] - (bmin[a] == 0.0f ? 1.0f : 0.0f) * 1e-8f;
            bmax[a] = bmax[a] + (bmax[a] == 0.0f ? 1.0f : 0.0f) * 1e-8f;
        }
        int32_t c_idx = idx0, w_idx = -(idx0 + 1), level = 0;
        for (;;) {
            if (!(w_idx != 0 || level == 0)) break;                           // (:218)
            const int32_t p_idx = level == 0 ? parents[c_idx + num] : parents[c_idx];
            uint32_t *node = nodes + 16 * (size_t)p_idx;
            uint32_t sibling;
            if (nt > 1) {
                sibling = __atomic_fetch_add(&node[7], 1u, __ATOMIC_ACQ_REL);
            } else {
                sibling = node[7]++;                                         // atomicAdd f_1 (:230)
            }
            if (sibling == 0) {                                              // (:233-243)
                node[0] = f32(bmin[0]); node[1] = f32(bmin[1]); node[2] = f32(bmin[2]);
                node[4] = f32(bmax[0]); node[5] = f32(bmax[1]); node[6] = f32(bmax[2]);
                node[3] = (uint32_t)w_idx;
                if (nt > 1) ready[p_idx].store(1, std::memory_order_release);
                break;
            }
            // second arrival: right slot, then merge with the left one (:245-271)
            node[8] = f32(bmin[0]); node[9] = f32(bmin[1]); node[10] = f32(bmin[2]);
            node[12] = f32(bmax[0]); node[13] = f32(bmax[1]); node[14] = f32(bmax[2]);
            node[11] = (uint32_t)w_idx;
            if (nt > 1)
                while (ready[p_idx].load(std::memory_order_acquire) == 0) { /* left writer is mid-store */ }
            for (int a = 0; a < 3; ++a) {
                bmin[a] = fmin_w(bmin[a], u2f(node[a]));
                bmax[a] = fmax_w(bmax[a], u2f(node[4 + a]));
            }
            c_idx = p_idx; w_idx = p_idx; level += 1;                         // (:273-277)
        }
    }
}

// Canonical form of a tree built by the arrival-order protocol: the Karras left child
// (the child at the lower split position: an internal child's index or a leaf's sorted
// position, since the children of split gamma are gamma and gamma + 1) goes in the left
// slot, f_1 = 2, f_2 = 0.  An N = 1 tree keeps its single arrival (f_1 = 1).
void oracle_canonicalize(uint32_t *nodes, uint32_t n) {
    if (n == 0) return;
    if (n == 1) { nodes[7] = 1; nodes[15] = 0; return; }
    for (uint64_t p = 0; p + 1 < n; ++p) {
        uint32_t *node = nodes + 16 * p;
        int32_t lc = (int32_t)node[3], rc = (int32_t)node[11];
        int32_t lpos = lc >= 0 ? lc : -(lc + 1);
        int32_t rpos = rc >= 0 ? rc : -(rc + 1);
        if (lpos > rpos) {
            for (int w = 0; w < 8; ++w) std::swap(node[w], node[8 + w]);
        }
        node[7] = 2; node[15] = 0;
    }
}

// rearrange_triangles (scripts/bvh/kernels/rearrange.js:162-169): o_tri[i] = i_tri[idx[i]],
// whole 48-byte records (pad words included).
void oracle_rearrange(const float *tri, const int32_t *idx, uint32_t n, float *out, int threads) {
#pragma omp parallel for schedule(static) num_threads(num_threads(threads))
    for (int64_t i = 0; i < (int64_t)n; ++i)
        std::memcpy(out + 12 * i, tri + 12 * (size_t)idx[i], 48);
}

// Indexed mesh -> 48-byte soup (pad words 0), the gather lvbh_build_indexed performs.
void oracle_gather_indexed(const float *xyz, const uint32_t *idx3, uint32_t n, float *tri) {
    for (uint64_t i = 0; i < n; ++i)
        for (int v = 0; v < 3; ++v) {
            const float *p = xyz + 3 * (size_t)idx3[3 * i + v];
            float *o = tri + 12 * i + 4 * v;
            o[0] = p[0]; o[1] = p[1]; o[2] = p[2]; o[3] = 0.0f;
        }
}

// build() (scripts/bvh/build-bvh.js:12-66) chained, canonical output.  bounds6 = NULL
// reduces the scene box over all vertices (oracle_scene_bounds).  Any output may be NULL.
// Returns 0.
int oracle_build(const float *tri, uint32_t n, const float *bounds6, int threads,
                 uint32_t *nodes_out, float *tris_out, int32_t *parents_out,
                 int32_t *perm_out, uint32_t *keys_out, float *bounds_used) {
    float b[6];
    if (bounds6) std::memcpy(b, bounds6, sizeof b); else oracle_scene_bounds(tri, n, b);
    if (bounds_used) std::memcpy(bounds_used, b, sizeof b);
    if (n == 0) return 0;
    std::vector<float> aabb((size_t)n * 8);
    std::vector<uint32_t> keys(n);
    std::vector<int32_t> perm(n), parents((size_t)2 * n);
    std::vector<uint32_t> nodes;
    oracle_aabb_zidx(tri, n, b, aabb.data(), keys.data(), threads);
    oracle_radix_sort(keys.data(), n, perm.data(), threads);
    oracle_radix_tree(keys.data(), n, parents.data(), threads);
    uint32_t *nd = nodes_out;
    if (!nd) { nodes.resize((size_t)16 * n); nd = nodes.data(); }
    oracle_up_pass(perm.data(), aabb.data(), parents.data(), n, nd, threads);
    oracle_canonicalize(nd, n);
    if (tris_out) oracle_rearrange(tri, perm.data(), n, tris_out, threads);
    if (parents_out) std::memcpy(parents_out, parents.data(), sizeof(int32_t) * 2 * (size_t)n);
    if (perm_out) std::memcpy(perm_out, perm.data(), sizeof(int32_t) * (size_t)n);
    if (keys_out) std::memcpy(keys_out, keys.data(), sizeof(uint32_t) * (size_t)n);
    return 0;
}

// ---- traversal (validation consumer) ---------------------------------------------------
// intersect_bvh / tri_intersect / aabb_intersect (scripts/pathtracer/pathtracer.js:495-584,
// 587-619, 621-628), returning the hit leaf's sorted position (the reference returns only
// the normal and distance) and the deepest stack used.  The stack holds 64 entries where
// the reference's holds 32 (:493); max_stack reports how deep each ray went.

struct V3 { float x, y, z; };
static inline V3 sub3(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross3(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

static float tri_intersect(V3 o, V3 d, const float *t) {
    V3 v0 = {t[0], t[1], t[2]}, v1 = {t[4], t[5], t[6]}, v2 = {t[8], t[9], t[10]};
    V3 v0v1 = sub3(v1, v0), v0v2 = sub3(v2, v0);
    V3 pvec = cross3(d, v0v2);
    float det = dot3(v0v1, pvec);
    if (std::fabs(det) < 1e-10f) return -1.0f;
    float i_det = 1.0f / det;
    V3 tvec = sub3(o, v0);
    float u = dot3(tvec, pvec) * i_det;
    if (u < 0.0f || u > 1.0f) return -1.0f;
    V3 qvec = cross3(tvec, v0v1);
    float v = dot3(d, qvec) * i_det;
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    return dot3(v0v2, qvec) * i_det;
}

static float aabb_intersect(V3 lo, V3 hi, V3 o, V3 d) {
    V3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    V3 f = {(hi.x - o.x) * inv.x, (hi.y - o.y) * inv.y, (hi.z - o.z) * inv.z};
    V3 nn = {(lo.x - o.x) * inv.x, (lo.y - o.y) * inv.y, (lo.z - o.z) * inv.z};
    V3 tmax = {fmax_w(f.x, nn.x), fmax_w(f.y, nn.y), fmax_w(f.z, nn.z)};
    V3 tmin = {fmin_w(f.x, nn.x), fmin_w(f.y, nn.y), fmin_w(f.z, nn.z)};
    float t0 = fmax_w(tmin.x, fmax_w(tmin.y, tmin.z));
    float t1 = fmin_w(tmax.x, fmin_w(tmax.y, tmax.z));
    return (t1 >= t0) ? ((t1 < 0.0f) ? -1e30f : t0) : -1e30f;
}

// One ray: o, d as given to intersect_bvh (d is nudged away from zero here, :501).  Returns the
// hit leaf's sorted position (-1 = miss) with its distance in *dist (-1 = miss) and the deepest
// stack in *deepest.
int32_t oracle_trace_one(const uint32_t *nodes, const float *tris, uint32_t n, const float *o_in,
                         const float *d_in, float *dist_out, uint32_t *deepest_out) {
    auto u2f = [](uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; };
    V3 o = {o_in[0], o_in[1], o_in[2]};
    V3 d = {d_in[0], d_in[1], d_in[2]};
    // d += vec3f(abs(d) < vec3f(.00001)) * vec3f(.00001)   (:501)
    d.x = d.x + (std::fabs(d.x) < 1e-5f ? 1.0f : 0.0f) * 1e-5f;
    d.y = d.y + (std::fabs(d.y) < 1e-5f ? 1.0f : 0.0f) * 1e-5f;
    d.z = d.z + (std::fabs(d.z) < 1e-5f ? 1.0f : 0.0f) * 1e-5f;
    float dist = 1e30f;
    int32_t prim = -1;
    int32_t stack[64];
    int32_t sp = 0, node_idx = 0;
    uint32_t deepest = 0;
    if (n == 0) sp = -1;
    while (sp >= 0) {
        if (node_idx < 0) {
            const int32_t leaf = -(node_idx + 1);
            float t = tri_intersect(o, d, tris + 12 * (size_t)leaf);
            if (t > 0.0f && t < dist) { dist = fmin_w(t, dist); prim = leaf; }
            sp -= 1;
            node_idx = sp >= 0 ? stack[sp] : 0;
        } else {
            const uint32_t *nd = nodes + 16 * (size_t)node_idx;
            V3 lmin = {u2f(nd[0]), u2f(nd[1]), u2f(nd[2])}, lmax = {u2f(nd[4]), u2f(nd[5]), u2f(nd[6])};
            V3 rmin = {u2f(nd[8]), u2f(nd[9]), u2f(nd[10])}, rmax = {u2f(nd[12]), u2f(nd[13]), u2f(nd[14])};
            int32_t lc = (int32_t)nd[3], rc = (int32_t)nd[11];
            float ld = aabb_intersect(lmin, lmax, o, d);
            float rd = aabb_intersect(rmin, rmax, o, d);
            bool lv = ld != -1e30f && ld < dist;
            bool rv = rd != -1e30f && rd < dist;
            if (lv && rv) {
                int32_t c, f;
                if (ld < rd) { c = lc; f = rc; } else { c = rc; f = lc; }
                if (sp < 64) stack[sp] = f;
                sp += 1;
                if ((uint32_t)sp > deepest) deepest = (uint32_t)sp;
                if (sp > 64) { sp = -1; break; }   // deeper than this restatement holds
                node_idx = c;
            } else if (lv) {
                node_idx = lc;
            } else if (rv) {
                node_idx = rc;
            } else {
                sp -= 1;
                node_idx = sp >= 0 ? stack[sp] : 0;
            }
        }
    }
    *dist_out = dist == 1e30f ? -1.0f : dist;
    if (deepest_out) *deepest_out = deepest;
    return dist == 1e30f ? -1 : prim;
}

void oracle_trace(const uint32_t *nodes, const float *tris, uint32_t n, const float *rays,
                  uint32_t num_rays, int32_t *hit_prim, float *hit_t, uint32_t *max_stack,
                  int threads) {
#pragma omp parallel for schedule(dynamic, 1024) num_threads(num_threads(threads))
    for (int64_t r = 0; r < (int64_t)num_rays; ++r) {
        const float *ry = rays + 8 * r;
        uint32_t deepest = 0;
        hit_prim[r] = oracle_trace_one(nodes, tris, n, ry, ry + 4, hit_t + r, &deepest);
        if (max_stack) max_stack[r] = deepest;
    }
}

}  // extern "C"
