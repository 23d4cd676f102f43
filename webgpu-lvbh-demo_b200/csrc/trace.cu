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
constexpr int kSmemStack = 32;  // the first entries of a ray's stack, in shared memory

// A ray's stack: entries 0 .. kSmemStack - 1 in shared memory, entry i of thread t at [i][t] (a
// warp's 32 entries of one depth in 32 banks); deeper entries (rare) in thread-local memory.
template <int NT>
struct RayStack {
    int32_t *s;     // &smem[0][threadIdx.x] of a [kSmemStack][NT] array
    int32_t *deep;  // kStack - kSmemStack entries
    __device__ __forceinline__ int32_t &operator[](int i) const {
        return i < kSmemStack ? s[i * NT] : deep[i - kSmemStack];
    }
};

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

// Where a leaf's three vertices come from: the 48-byte sorted soup, or the indexed leaf format
// (three vertex indices per sorted leaf into 16-byte vertex rows; an index past the buffer
// reads row 0).
struct SoupTris {
    const float4 *tris;
    __device__ __forceinline__ void get(int leaf, float4 &a, float4 &b, float4 &c) const {
        const float4 *t = tris + 3ull * leaf;
        a = __ldg(t);
        b = __ldg(t + 1);
        c = __ldg(t + 2);
    }
};
struct MeshTris {
    const float4 *verts;
    const uint32_t *sidx;
    uint32_t nverts;
    __device__ __forceinline__ void get(int leaf, float4 &a, float4 &b, float4 &c) const {
        const uint32_t *r = sidx + 3ull * leaf;
        const uint32_t i0 = __ldg(r), i1 = __ldg(r + 1), i2 = __ldg(r + 2);
        a = __ldg(verts + (i0 < nverts ? i0 : 0u));
        b = __ldg(verts + (i1 < nverts ? i1 : 0u));
        c = __ldg(verts + (i2 < nverts ? i2 : 0u));
    }
};

template <class Tris>
__device__ float tri_intersect(F3 o, F3 d, const Tris &tr, int leaf) {
    float4 a, b, c;
    tr.get(leaf, a, b, c);
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
    const float4 ro = rays[2ull * r], rd = rays[2ull * r + 1];
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
template <class Tris, class Stack>
__device__ __forceinline__ bool ray_step(RayState &st, const Stack &stack, const float4 *__restrict__ nodes,
                                         const Tris &tris, uint32_t n) {
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
        const float t = tri_intersect(st.o, st.d, tris, leaf);
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
template <class Tris>
__global__ void __launch_bounds__(128) k_trace(const float4 *__restrict__ nodes, Tris tris, uint32_t n,
                                               const float4 *__restrict__ rays, uint32_t num_rays,
                                               int32_t *__restrict__ hit_prim,
                                               float *__restrict__ hit_t,
                                               uint32_t *__restrict__ max_stack,
                                               uint32_t *__restrict__ counter) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    // the first kSmemStack entries in shared memory (1,515 -> 1,580 M rays/s on the 2 M sphere)
    __shared__ int32_t sstack[kSmemStack][128];
    int32_t deep[kStack - kSmemStack];
    const RayStack<128> stack{&sstack[0][threadIdx.x], deep};
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

// ---- path-trace bounce (sample(), pathtracer.js:360-392 -> main / ptStep, :630-713) ----------
// The WGSL leaves sin, cos, pow and normalize to the implementation; these definitions fix
// them: normalize(v) = v / sqrt(dot(v, v)) (IEEE square root and divisions), sin / cos by
// Cody-Waite reduction over pi/2 (three-part float split, k * C1 and k * C2 exact) and Taylor
// polynomials to degree 11 / 10, pow(.3, 2.2) a host constant.  Every operation is an
// explicitly rounded intrinsic, so a CPU restatement in the same order gives the same bits.

__device__ __forceinline__ F3 add3(F3 a, F3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ F3 mul3(F3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ F3 normalize3(F3 v) {
    const float len = __fsqrt_rn(dot3(v, v));
    return {__fdiv_rn(v.x, len), __fdiv_rn(v.y, len), __fdiv_rn(v.z, len)};
}
__device__ __forceinline__ F3 to_world(F3 vx, F3 vy, F3 vz, F3 w) {
    return add3(add3(mul3(vx, w.x), mul3(vy, w.y)), mul3(vz, w.z));
}
__device__ __forceinline__ F3 ortho3(F3 v) {
    if (fabsf(v.x) > fabsf(v.y)) return {-v.y, v.x, 0.0f};
    return {0.0f, -v.z, v.y};
}

__device__ __forceinline__ void pt_sincos(float theta, float &s_out, float &c_out) {
    const float kTwoOverPi = 0x1.45f306p-1f;
    const float C1 = 0x1.92p+0f, C2 = 0x1.fb544p-12f, C3 = 0x1.0b4612p-34f;
    const int k = __float2int_rn(__fmul_rn(theta, kTwoOverPi));
    const float kf = __int2float_rn(k);
    const float r = __fsub_rn(__fsub_rn(__fsub_rn(theta, __fmul_rn(kf, C1)), __fmul_rn(kf, C2)), __fmul_rn(kf, C3));
    const float r2 = __fmul_rn(r, r);
    float ps = __fadd_rn(0x1.71de3ap-19f, __fmul_rn(r2, -0x1.ae6456p-26f));
    ps = __fadd_rn(-0x1.a01a02p-13f, __fmul_rn(r2, ps));
    ps = __fadd_rn(0x1.111112p-7f, __fmul_rn(r2, ps));
    ps = __fadd_rn(-0x1.555556p-3f, __fmul_rn(r2, ps));
    const float s = __fadd_rn(r, __fmul_rn(__fmul_rn(r, r2), ps));
    float pc = __fadd_rn(0x1.a01a02p-16f, __fmul_rn(r2, -0x1.27e4fcp-22f));
    pc = __fadd_rn(-0x1.6c16c2p-10f, __fmul_rn(r2, pc));
    pc = __fadd_rn(0x1.555556p-5f, __fmul_rn(r2, pc));
    pc = __fadd_rn(-0x1p-1f, __fmul_rn(r2, pc));
    const float c = __fadd_rn(1.0f, __fmul_rn(r2, pc));
    switch (k & 3) {
        case 0: s_out = s; c_out = c; break;
        case 1: s_out = c; c_out = -s; break;
        case 2: s_out = -s; c_out = -c; break;
        default: s_out = -c; c_out = s; break;
    }
}

// baseHash (:752-756).
__device__ __forceinline__ uint32_t base_hash(uint32_t px, uint32_t py) {
    const uint32_t p2x = 1103515245u * ((px >> 1) ^ py);
    const uint32_t p2y = 1103515245u * ((py >> 1) ^ px);
    const uint32_t h32 = 1103515245u * (p2x ^ (p2y >> 3));
    return h32 ^ (h32 >> 16);
}

// rand2 (:757-761).
__device__ __forceinline__ void rand2(float seed, float &rx, float &ry) {
    const uint32_t n = base_hash(__float_as_uint(__fadd_rn(seed, 1.0f)), __float_as_uint(__fadd_rn(seed, 2.0f)));
    rx = __fdiv_rn(__uint2float_rn(n & 0x7fffffffu), 2147483648.0f);
    ry = __fdiv_rn(__uint2float_rn((n * 48271u) & 0x7fffffffu), 2147483648.0f);
}

// One pixel's path between bounces (the four state images' texels).
struct PixelPath {
    F3 o, d, b;
    float4 t;
    float seed, bounces;
    uint32_t px;
};

// ptStep up to the traversal (:656-674): a new path draws its camera ray.
__device__ __forceinline__ void pt_begin(PixelPath &pp, const float4 *__restrict__ in, size_t plane, uint32_t px,
                                         const PtFrame &f) {
    pp.px = px;
    const uint32_t cx = px % f.width, cy = px / f.width;
    float4 o4 = make_float4(0.f, 0.f, 0.f, 0.f), d4 = o4, t4 = o4, b4 = o4;
    if (f.rst == 0.0f) {
        o4 = __ldcs(in + px);
        d4 = __ldcs(in + plane + px);
        t4 = __ldcs(in + 2 * plane + px);
        b4 = __ldcs(in + 3 * plane + px);
    }
    pp.o = {o4.x, o4.y, o4.z};
    pp.d = {d4.x, d4.y, d4.z};
    pp.b = {b4.x, b4.y, b4.z};
    pp.t = t4;
    pp.seed = o4.w;
    pp.bounces = d4.w;
    const bool new_path = pp.b.x == 0.0f && pp.b.y == 0.0f && pp.b.z == 0.0f;
    if (new_path && t4.w == 0.0f)
        pp.seed = __fadd_rn(__fdiv_rn(__uint2float_rn(base_hash(cx, cy)), 4294967296.0f), 0.008f);
    if (new_path) {
        float rx, ry;
        rand2(pp.seed, rx, ry);
        float sx = __fdiv_rn(__fadd_rn(__uint2float_rn(cx), rx), f.sw_x);
        float sy = __fdiv_rn(__fadd_rn(__uint2float_rn(cy), ry), f.sw_y);
        sx = __fsub_rn(__fmul_rn(sx, 2.0f), 1.0f);
        sy = -__fsub_rn(__fmul_rn(sy, 2.0f), 1.0f);
        const F3 local = {__fmul_rn(__fmul_rn(f.aspect, sx), f.sinfov), 1.0f, __fmul_rn(sy, f.sinfov)};
        const F3 pos = {f.pos[0], f.pos[1], f.pos[2]}, lat = {f.lat[0], f.lat[1], f.lat[2]};
        const F3 forward = normalize3(sub3(lat, pos));
        const F3 right = normalize3(F3{forward.y, -forward.x, 0.0f});
        const F3 up = cross3(right, forward);
        pp.o = pos;
        pp.d = to_world(right, forward, up, normalize3(local));
        pp.seed = __fadd_rn(pp.seed, 2.0f);
        pp.b = {1.0f, 1.0f, 1.0f};
    }
}

// ptStep after the traversal (:675-712) and the texel stores.
template <class Tris>
__device__ __forceinline__ void pt_end(PixelPath &pp, const RayState &st, const Tris &tris,
                                       float4 *__restrict__ out, size_t plane, const PtFrame &f) {
    const float eps = 0.0001f, two_pi = 0x1.921fb6p+2f;
    F3 b = pp.b;
    float4 t = pp.t;
    float seed = pp.seed, bounces = pp.bounces;
    F3 o = pp.o, d = pp.d;
    if (st.dist != 1e30f) {
        float4 a, bb, c;
        tris.get(st.prim, a, bb, c);
        const F3 v0 = {a.x, a.y, a.z}, v1 = {bb.x, bb.y, bb.z}, v2 = {c.x, c.y, c.z};
        F3 norm = normalize3(cross3(sub3(v1, v0), sub3(v2, v0)));
        if (!(dot3(st.d, F3{-norm.x, -norm.y, -norm.z}) > 0.0f)) norm = {-norm.x, -norm.y, -norm.z};
        const F3 o1 = normalize3(ortho3(norm));
        const F3 o2 = normalize3(cross3(o1, norm));
        o = add3(o, mul3(d, st.dist));
        float r2x, r2y;
        rand2(seed, r2x, r2y);
        const float rr = __fsqrt_rn(r2x > 0.0f ? r2x : 0.0f);
        float sn, cs;
        pt_sincos(__fmul_rn(two_pi, r2y), sn, cs);
        const float dx = __fmul_rn(rr, cs), dy = __fmul_rn(rr, sn);
        const float zz = __fsub_rn(__fsub_rn(1.0f, __fmul_rn(dx, dx)), __fmul_rn(dy, dy));
        const F3 wi = {dx, dy, __fsqrt_rn(zz > 0.0f ? zz : 0.0f)};
        seed = __fadd_rn(seed, 2.0f);
        b = mul3(b, f.powc);
        o = add3(o, mul3(mul3(norm, 1.01f), eps));
        d = to_world(o1, o2, norm, wi);
        if (bounces > 3.0f) {
            const float q1 = __fsub_rn(1.0f, b.y), q = 0.05f > q1 ? 0.05f : q1;
            float ux, uy;
            rand2(seed, ux, uy);
            if (ux < q) {
                b = {0.0f, 0.0f, 0.0f};
            } else {
                const float keep = __fsub_rn(1.0f, q);
                b = {__fdiv_rn(b.x, keep), __fdiv_rn(b.y, keep), __fdiv_rn(b.z, keep)};
            }
            seed = __fadd_rn(seed, 2.0f);
        }
        if (b.x == 0.0f && b.y == 0.0f && b.z == 0.0f) {
            t = make_float4(__fadd_rn(t.x, 0.0f), __fadd_rn(t.y, 0.0f), __fadd_rn(t.z, 0.0f), __fadd_rn(t.w, 1.0f));
            bounces = -1.0f;
        }
    } else {
        t = make_float4(__fadd_rn(t.x, __fmul_rn(b.x, 8.0f)), __fadd_rn(t.y, __fmul_rn(b.y, 8.0f)),
                        __fadd_rn(t.z, __fmul_rn(b.z, 8.0f)), __fadd_rn(t.w, 1.0f));
        bounces = -1.0f;
        b = {0.0f, 0.0f, 0.0f};
    }
    const uint32_t px = pp.px;
    __stcs(out + px, make_float4(o.x, o.y, o.z, seed));
    __stcs(out + plane + px, make_float4(d.x, d.y, d.z, __fadd_rn(bounces, 1.0f)));
    __stcs(out + 2 * plane + px, t);
    __stcs(out + 3 * plane + px, make_float4(b.x, b.y, b.z, 1.0f));
}

// One bounce of every pixel: persistent warps fetch pixels from *counter as lanes finish (the
// traversal's dynamic fetch), each pixel's walk exactly the reference's.
template <class Tris>
__global__ void __launch_bounds__(128) k_pt_step(const float4 *__restrict__ nodes, Tris tris,
                                                 uint32_t n, const float4 *__restrict__ in, float4 *__restrict__ out,
                                                 PtFrame f, uint32_t *__restrict__ counter) {
    const int lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint32_t num = f.width * f.height;
    const size_t plane = num;
    // thread-local stack: this kernel's node fetches gain more from the L1 it would share with
    // a shared-memory stack (0.666 -> 0.700 ms per 1080p bounce with one) than the stack does
    int32_t stack_mem[kStack];
    int32_t *const stack = stack_mem;
    RayState st;
    PixelPath pp;
    bool have = false, exhausted = false;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !have);
        if (!exhausted && __popc(idle) >= 8) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(counter, (uint32_t)__popc(idle));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base + __popc(idle) >= num) exhausted = true;
            if (!have) {
                const uint32_t my = base + __popc(idle & lt);
                if (my < num) {
                    pt_begin(pp, in, plane, my, f);
                    const float4 ray[2] = {make_float4(pp.o.x, pp.o.y, pp.o.z, 0.f),
                                           make_float4(pp.d.x, pp.d.y, pp.d.z, 0.f)};
                    ray_init(st, ray, 0, n);
                    have = true;
                }
            }
        } else if (exhausted && idle == 0xFFFFFFFFu) {
            break;
        }
        if (have && !ray_step(st, stack, nodes, tris, n)) {
            pt_end(pp, st, tris, out, plane, f);
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
    if (!per_sm && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<SoupTris>, 128, 0) != cudaSuccess ||
                    per_sm < 1)) {
        cudaGetLastError();
        per_sm = 4;
    }
    const uint32_t want = (num_rays + 127) / 128, cap = (uint32_t)(sm_count() * per_sm);
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    k_trace<<<want < cap ? want : cap, 128, 0, s>>>(nodes, SoupTris{tris}, n, rays, num_rays, hit_prim, hit_t,
                                                    max_stack, counter);
}

void launch_trace_mesh(const float4 *nodes, const float4 *verts, uint32_t num_verts, const uint32_t *sidx, uint32_t n,
                       const float4 *rays, uint32_t num_rays, int32_t *hit_prim, float *hit_t,
                       uint32_t *max_stack, uint32_t *counter, cudaStream_t s) {
    if (num_rays == 0) return;
    static int per_sm = 0;
    if (!per_sm && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<MeshTris>, 128, 0) != cudaSuccess ||
                    per_sm < 1)) {
        cudaGetLastError();
        per_sm = 4;
    }
    const uint32_t want = (num_rays + 127) / 128, cap = (uint32_t)(sm_count() * per_sm);
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    k_trace<<<want < cap ? want : cap, 128, 0, s>>>(nodes, MeshTris{verts, sidx, num_verts}, n, rays, num_rays,
                                                    hit_prim, hit_t, max_stack, counter);
}

void launch_pt_step(const float4 *nodes, const float4 *tris, uint32_t n, const float4 *state_in,
                    float4 *state_out, const PtFrame &f, uint32_t *counter, cudaStream_t s) {
    const uint32_t num = f.width * f.height;
    if (num == 0) return;
    static int per_sm = 0;
    if (!per_sm && (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pt_step<SoupTris>, 128, 0) != cudaSuccess ||
                    per_sm < 1)) {
        cudaGetLastError();
        per_sm = 4;
    }
    const uint32_t want = (num + 127) / 128, cap = (uint32_t)(sm_count() * per_sm);
    cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    k_pt_step<<<want < cap ? want : cap, 128, 0, s>>>(nodes, SoupTris{tris}, n, state_in, state_out, f, counter);
}

}  // namespace lvbh
