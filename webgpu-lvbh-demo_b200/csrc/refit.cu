// refit.cu - K4: leaf gather, triangle rearrange and bottom-up box refit (sm_100a).
//
// Fuses rearrange_triangles (scripts/bvh/kernels/rearrange.js:162-169) with bvh_upward_pass
// (scripts/bvh/kernels/bvh-up-pass.js:200-280).  One thread per leaf (sorted position k):
//
//   * gathers triangle perm[k] (3 x 16-byte loads), writes it to the output soup at k
//     (o_tri[k] = i_tri[perm[k]], pad words included) and takes its box from the same
//     registers - the reference reads a separate per-triangle AABB buffer instead;
//   * nudges exactly-zero box components by 1e-8 as the reference does (:209-210);
//   * climbs the parent links.  At each parent it writes its own 32-byte half of the node
//     record (box + child link + sync word), fences, and exchanges the build's epoch into the
//     parent's arrival word.  The first arrival stops there; the second - which sees the
//     epoch already present - reads its sibling's half back from L2, merges the two boxes with
//     exact min/max and climbs on.  The reference instead lets the first arrival write the
//     left slot and has the second spin until no component of it reads 0.0; here nothing
//     waits, so the kernel cannot hang, and each climb is bounded by the deepest tree a
//     32-bit key plus 32-bit index tie-break can produce.
//   * slots are in canonical Karras order: a node is its parent's left child when it covers
//     the lower key range.  For leaf k that is delta(k, k+1) > delta(k, k-1); for internal
//     node p (whose index is one end of its range) it is d_p = -1, i.e.
//     delta(p, p-1) > delta(p, p+1).
//
// The epoch (written by K3) makes the arrival words reusable without clearing them: a word
// from an older build never equals the current epoch.
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

constexpr int kMaxClimb = 96;  // a valid tree is at most 64 levels deep

__global__ void __launch_bounds__(256) k_refit(const float4 *__restrict__ tri,
                                               const uint32_t *__restrict__ perm,
                                               const uint32_t *__restrict__ keys,
                                               const int32_t *__restrict__ parents, int n,
                                               float4 *__restrict__ otri, float4 *nodes,
                                               uint32_t *arrive, const uint32_t *epoch_p,
                                               Control *ctl) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n) return;
    uint32_t ti = __ldg(perm + k);
    if (ti >= (uint32_t)n) {  // only after an upstream failure; keep every access in bounds
        atomicOr(&ctl->err, ERR_CLIMB);
        ti = 0;
    }
    const float4 a = __ldg(tri + 3ull * ti);
    const float4 b = __ldg(tri + 3ull * ti + 1);
    const float4 c = __ldg(tri + 3ull * ti + 2);
    st_stream(otri + 3ull * k, a);
    st_stream(otri + 3ull * k + 1, b);
    st_stream(otri + 3ull * k + 2, c);

    float mnx = fminf(a.x, fminf(b.x, c.x)), mny = fminf(a.y, fminf(b.y, c.y)),
          mnz = fminf(a.z, fminf(b.z, c.z));
    float mxx = fmaxf(a.x, fmaxf(b.x, c.x)), mxy = fmaxf(a.y, fmaxf(b.y, c.y)),
          mxz = fmaxf(a.z, fmaxf(b.z, c.z));
    // min - (min == 0) * 1e-8f and max + (max == 0) * 1e-8f: exactly -+1e-8f at zero
    mnx = mnx == 0.0f ? -1e-8f : mnx; mny = mny == 0.0f ? -1e-8f : mny; mnz = mnz == 0.0f ? -1e-8f : mnz;
    mxx = mxx == 0.0f ? 1e-8f : mxx;  mxy = mxy == 0.0f ? 1e-8f : mxy;  mxz = mxz == 0.0f ? 1e-8f : mxz;

    if (n == 1) {  // one leaf, one arrival at node 0: left slot only, f_1 = 1
        nodes[0] = make_float4(mnx, mny, mnz, __int_as_float(-1));
        nodes[1] = make_float4(mxx, mxy, mxz, __int_as_float(1));
        nodes[2] = make_float4(0.f, 0.f, 0.f, 0.f);
        nodes[3] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    if (k == 0) {  // record N-1 is never a node; the reference leaves it zero
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 *last = nodes + 4ull * (n - 1);
        last[0] = z; last[1] = z; last[2] = z; last[3] = z;
    }
    const uint32_t epoch = *epoch_p;
    bool left = delta(keys, n, k, k + 1) > delta(keys, n, k, k - 1);
    int p = __ldg(parents + n + k);
    int child = -(k + 1);
    for (int level = 0; level < kMaxClimb; ++level) {
        if ((unsigned)p >= (unsigned)(n - 1)) break;  // not an internal node: malformed links
        float4 *nd = nodes + 4ull * p;
        const int own = left ? 0 : 2;
        nd[own] = make_float4(mnx, mny, mnz, __int_as_float(child));
        nd[own + 1] = make_float4(mxx, mxy, mxz, __int_as_float(left ? 2 : 0));
        __threadfence();
        if (atomicExch(arrive + p, epoch) != epoch) return;  // first arrival
        __threadfence();
        const float4 smn = __ldcg(nd + (2 - own));
        const float4 smx = __ldcg(nd + (3 - own));
        mnx = fminf(mnx, smn.x); mny = fminf(mny, smn.y); mnz = fminf(mnz, smn.z);
        mxx = fmaxf(mxx, smx.x); mxy = fmaxf(mxy, smx.y); mxz = fmaxf(mxz, smx.z);
        if (p == 0) return;
        child = p;
        left = delta(keys, n, p, p - 1) > delta(keys, n, p, p + 1);
        p = __ldg(parents + p);
    }
    atomicOr(&ctl->err, ERR_CLIMB);
}

}  // namespace

void launch_refit(const float4 *tri, const uint32_t *perm, const uint32_t *keys,
                  const int32_t *parents, uint32_t n, float4 *otri, float4 *nodes,
                  uint32_t *arrive, const uint32_t *epoch, Control *ctl, cudaStream_t s) {
    if (n == 0) return;
    k_refit<<<(n + 255) / 256, 256, 0, s>>>(tri, perm, keys, parents, (int)n, otri, nodes,
                                            arrive, epoch, ctl);
}

}  // namespace lvbh
