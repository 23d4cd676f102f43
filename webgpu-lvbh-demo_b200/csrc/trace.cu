// trace.cu - K5: closest-hit traversal of a built tree (validation consumer, sm_100a).
//
// Restates intersect_bvh (scripts/pathtracer/pathtracer.js:495-584), tri_intersect
// (:587-619) and aabb_intersect (:621-628) - the consumer whose node and triangle layouts the
// build must keep - and additionally returns the hit triangle's sorted position and the
// deepest stack each ray used.  Every f32 operation is an explicitly rounded intrinsic (no
// contraction into FMA), division is correctly rounded and min/max are `a < b ? a : b`, so a
// CPU restatement with the same operation order returns bit-identical distances.
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

constexpr int kStack = 64;  // the reference's private stack holds 32 (:493)

struct F3 { float x, y, z; };
__device__ __forceinline__ float wmin(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float wmax(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) {
    return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ float dot3(F3 a, F3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}

__device__ float tri_intersect(F3 o, F3 d, const float4 *t) {
    const float4 a = __ldg(t), b = __ldg(t + 1), c = __ldg(t + 2);
    const F3 v0 = {a.x, a.y, a.z}, v1 = {b.x, b.y, b.z}, v2 = {c.x, c.y, c.z};
    const F3 v0v1 = sub3(v1, v0), v0v2 = sub3(v2, v0);
    const F3 pvec = cross3(d, v0v2);
    const float det = dot3(v0v1, pvec);
    if (fabsf(det) < 1e-10f) return -1.0f;
    const float i_det = __fdiv_rn(1.0f, det);
    const F3 tvec = sub3(o, v0);
    const float u = __fmul_rn(dot3(tvec, pvec), i_det);
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const F3 qvec = cross3(tvec, v0v1);
    const float v = __fmul_rn(dot3(d, qvec), i_det);
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return -1.0f;
    return __fmul_rn(dot3(v0v2, qvec), i_det);
}

__device__ __forceinline__ float aabb_intersect(F3 lo, F3 hi, F3 o, F3 inv) {
    const float fx = __fmul_rn(__fsub_rn(hi.x, o.x), inv.x), nx = __fmul_rn(__fsub_rn(lo.x, o.x), inv.x);
    const float fy = __fmul_rn(__fsub_rn(hi.y, o.y), inv.y), ny = __fmul_rn(__fsub_rn(lo.y, o.y), inv.y);
    const float fz = __fmul_rn(__fsub_rn(hi.z, o.z), inv.z), nz = __fmul_rn(__fsub_rn(lo.z, o.z), inv.z);
    const float t0 = wmax(wmin(fx, nx), wmax(wmin(fy, ny), wmin(fz, nz)));
    const float t1 = wmin(wmax(fx, nx), wmin(wmax(fy, ny), wmax(fz, nz)));
    return (t1 >= t0) ? ((t1 < 0.0f) ? -1e30f : t0) : -1e30f;
}

// One ray's traversal state.
struct RayState {
    F3 o, d, inv;
    float dist;
    int32_t prim;
    int sp, node_idx;
    uint32_t deepest;
    uint32_t visits;  // node visits so far: a valid tree needs fewer than 2 N
};

__device__ __forceinline__ void ray_init(RayState &st, const float4 *__restrict__ rays, uint32_t r,
                                         uint32_t n) {
    const float4 ro = __ldg(rays + 2ull * r), rd = __ldg(rays + 2ull * r + 1);
    st.o = {ro.x, ro.y, ro.z};
    F3 d = {rd.x, rd.y, rd.z};
    // d += vec3f(abs(d) < vec3f(.00001)) * vec3f(.00001)   (:501)
    d.x = fabsf(d.x) < 1e-5f ? __fadd_rn(d.x, 1e-5f) : d.x;
    d.y = fabsf(d.y) < 1e-5f ? __fadd_rn(d.y, 1e-5f) : d.y;
    d.z = fabsf(d.z) < 1e-5f ? __fadd_rn(d.z, 1e-5f) : d.z;
    st.d = d;
    // aabb_intersect's `1. / d`, hoisted: the same value for every box
    st.inv = {__fdiv_rn(1.0f, d.x), __fdiv_rn(1.0f, d.y), __fdiv_rn(1.0f, d.z)};
    st.dist = 1e30f;
    st.prim = -1;
    st.sp = n == 0 ? -1 : 0;
    st.node_idx = 0;
    st.deepest = 0;
    st.visits = 0;
}

// One node visit of the reference's loop (pathtracer.js:505-581): a leaf is tested, an internal
// node's children are tested and the nearer valid one is taken with the farther pushed.
// Returns false once the ray's stack is empty.
__device__ __forceinline__ bool ray_step(RayState &st, int32_t *stack, const float4 *__restrict__ nodes,
                                         const float4 *__restrict__ tris, uint32_t n) {
    if (st.sp < 0) return false;
    const int node_idx = st.node_idx;
    if ((node_idx < 0 ? (uint32_t)(-(node_idx + 1)) >= n : (uint32_t)node_idx >= n) ||
        ++st.visits > 2u * n + 64u) {
        st.sp = -1;  // a link outside the tree or a cycle: stop this ray (never on a built tree)
        st.deepest = 0xFFFFFFFFu;
        return false;
    }
    if (node_idx < 0) {
        const int leaf = -(node_idx + 1);
        const float t = tri_intersect(st.o, st.d, tris + 3ull * leaf);
        if (t > 0.0f && t < st.dist) { st.dist = wmin(t, st.dist); st.prim = leaf; }
        st.sp -= 1;
        st.node_idx = st.sp >= 0 ? stack[st.sp] : 0;
    } else {
        const float4 *nd = nodes + 4ull * node_idx;
        const float4 l0 = __ldg(nd), l1 = __ldg(nd + 1), r0 = __ldg(nd + 2), r1 = __ldg(nd + 3);
        const float ld = aabb_intersect({l0.x, l0.y, l0.z}, {l1.x, l1.y, l1.z}, st.o, st.inv);
        const float rdist = aabb_intersect({r0.x, r0.y, r0.z}, {r1.x, r1.y, r1.z}, st.o, st.inv);
        const int lc = __float_as_int(l0.w), rc = __float_as_int(r0.w);
        const bool lv = ld != -1e30f && ld < st.dist;
        const bool rv = rdist != -1e30f && rdist < st.dist;
        if (lv && rv) {
            const bool near_left = ld < rdist;
            if (st.sp >= kStack) { st.sp = -1; st.deepest = kStack + 1; return false; }
            stack[st.sp] = near_left ? rc : lc;
            st.sp += 1;
            st.deepest = max(st.deepest, (uint32_t)st.sp);
            st.node_idx = near_left ? lc : rc;
        } else if (lv) {
            st.node_idx = lc;
        } else if (rv) {
            st.node_idx = rc;
        } else {
            st.sp -= 1;
            st.node_idx = st.sp >= 0 ? stack[st.sp] : 0;
        }
    }
    return st.sp >= 0;
}

// Persistent traversal: each lane takes a new ray as soon as its current one is done (a warp
// refills its idle lanes from a global counter once a quarter of them are idle), so a warp is
// not held by its slowest ray.  Each ray's own walk is exactly the reference's.
__global__ void __launch_bounds__(128) k_trace(const float4 *__restrict__ nodes,
                                               const float4 *__restrict__ tris, uint32_t n,
                                               const float4 *__restrict__ rays, uint32_t num_rays,
                                               int32_t *__restrict__ hit_prim,
                                               float *__restrict__ hit_t,
                                               uint32_t *__restrict__ max_stack,
                                               uint32_t *__restrict__ counter) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    int32_t stack[kStack];
    RayState st;
    bool have = false, exhausted = false;
    uint32_t r = 0;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !have);
        if (!exhausted && __popc(idle) >= 8) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(counter, (uint32_t)__popc(idle));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base + __popc(idle) >= num_rays) exhausted = true;
            if (!have) {
                const uint32_t my = base + __popc(idle & lt);
                if (my < num_rays) {
                    r = my;
                    ray_init(st, rays, r, n);
                    have = true;
                }
            }
        } else if (exhausted && idle == 0xFFFFFFFFu) {
            break;
        }
        if (have && !ray_step(st, stack, nodes, tris, n)) {
            hit_prim[r] = st.dist == 1e30f ? -1 : st.prim;
            hit_t[r] = st.dist == 1e30f ? -1.0f : st.dist;
            if (max_stack) max_stack[r] = st.deepest;
            have = false;
        }
    }
}

}  // namespace

void launch_trace(const float4 *nodes, const float4 *tris, uint32_t n, const float4 *rays,
                  uint32_t num_rays, int32_t *hit_prim, float *hit_t, uint32_t *max_stack,
                  uint32_t *counter, cudaStream_t s) {
    if (num_rays == 0) return;
    static int per_sm = 0;
    if (!per_sm && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace, 128, 0) != cudaSuccess ||
                    per_sm < 1)) {
        cudaGetLastError();
        per_sm = 4;
    }
    const uint32_t want = (num_rays + 127) / 128, cap = (uint32_t)(sm_count() * per_sm);
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    k_trace<<<want < cap ? want : cap, 128, 0, s>>>(nodes, tris, n, rays, num_rays, hit_prim, hit_t,
                                                    max_stack, counter);
}

}  // namespace lvbh
