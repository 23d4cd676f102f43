// pt_oracle.cpp - CPU restatement of the reference's path-trace bounce.  TEST INFRASTRUCTURE ONLY.
//
// Part of the parity oracle (oracle/liblvbh_oracle.so): only tests/ and bench.py's CPU-baseline
// arm use it, as the checker; the product library never does.
//
// Restates one call of sample() (scripts/pathtracer/pathtracer.js:360-392): the compute shader
// main (:630-653) runs ptStep (:655-713) once per pixel over the four rgba32f state images
// (o = origin + seed, d = direction + bounce count, t = accumulated radiance + sample count,
// b = throughput + 1), with getCameraRay (:720-734), intersect_bvh (:495-584, through
// oracle_trace_one), lambertDiffuse (:715-718), cosineSampleHemisphere / uniformSampleDisk
// (:763-772), ortho / toWorld (:736-749) and the hashes baseHash / rand2 (:752-761).
//
// The WGSL leaves the precision of sin, cos, pow and normalize to the implementation; this
// restatement fixes them, and the device kernel uses the same definitions operation for
// operation, so both give the same bits:
//   normalize(v) = v / sqrt(dot(v, v)), each component one IEEE division;
//   sin / cos    = Cody-Waite reduction by pi/2 (three-part float split) and Taylor polynomials
//                  to degree 11 / 10 on [-pi/4, pi/4] (pt_sincos below), within 2 ulp;
//   pow(.3, 2.2) = the float nearest to 0.3f^2.2f (a host constant, `powc`);
//   sinfov and aspect, which the shader bakes in as constants, are host constants too.
// Every float operation is IEEE single precision without contraction (built with
// -ffp-contract=off), in the shader's order.
//
// Parity status: unpinned against a run of the reference (its shader needs a browser WebGPU).

#include <cmath>
#include <cstdint>
#include <cstring>

extern "C" int32_t oracle_trace_one(const uint32_t *nodes, const float *tris, uint32_t n, const float *o_in,
                                    const float *d_in, float *dist_out, uint32_t *deepest_out);

namespace {

struct V3 {
    float x, y, z;
};

inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 normalize(V3 v) {
    const float len = std::sqrt(dot(v, v));
    return {v.x / len, v.y / len, v.z / len};
}
inline V3 to_world(V3 vx, V3 vy, V3 vz, V3 w) { return add(add(mul(vx, w.x), mul(vy, w.y)), mul(vz, w.z)); }
inline V3 ortho(V3 v) {
    if (std::fabs(v.x) > std::fabs(v.y)) return {-v.y, v.x, 0.0f};
    return {0.0f, -v.z, v.y};
}

// sin and cos of theta (|theta| small multiples of pi): k = nearest integer to theta * 2/pi,
// r = theta - k pi/2 with pi/2 = C1 + C2 + C3 (C1, C2 short enough that k * C1 and k * C2 are
// exact), Taylor polynomials of sin and cos at r, then the quadrant k mod 4.
void pt_sincos(float theta, float *s_out, float *c_out) {
    const float kTwoOverPi = 0x1.45f306p-1f;
    const float C1 = 0x1.92p+0f, C2 = 0x1.fb544p-12f, C3 = 0x1.0b4612p-34f;
    const int k = (int)std::nearbyint(theta * kTwoOverPi);
    const float kf = (float)k;
    const float r = ((theta - kf * C1) - kf * C2) - kf * C3;
    const float r2 = r * r;
    const float s = r + (r * r2) * (-0x1.555556p-3f + r2 * (0x1.111112p-7f + r2 * (-0x1.a01a02p-13f +
                                    r2 * (0x1.71de3ap-19f + r2 * -0x1.ae6456p-26f))));
    const float c = 1.0f + r2 * (-0x1p-1f + r2 * (0x1.555556p-5f + r2 * (-0x1.6c16c2p-10f +
                                 r2 * (0x1.a01a02p-16f + r2 * -0x1.27e4fcp-22f))));
    switch (k & 3) {
        case 0: *s_out = s; *c_out = c; break;
        case 1: *s_out = c; *c_out = -s; break;
        case 2: *s_out = -s; *c_out = -c; break;
        default: *s_out = -c; *c_out = s; break;
    }
}

// baseHash (:752-756): integer hash of a pair.
inline uint32_t base_hash(uint32_t px, uint32_t py) {
    const uint32_t p2x = 1103515245u * ((px >> 1) ^ py);
    const uint32_t p2y = 1103515245u * ((py >> 1) ^ px);
    const uint32_t h32 = 1103515245u * (p2x ^ (p2y >> 3));
    return h32 ^ (h32 >> 16);
}

inline uint32_t bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// rand2 (:757-761): two uniforms in [0, 1] from the seed.
inline void rand2(float seed, float *rx, float *ry) {
    const uint32_t n = base_hash(bits(seed + 1.0f), bits(seed + 2.0f));
    const uint32_t zx = n, zy = n * 48271u;
    *rx = (float)(zx & 0x7fffffffu) / 2147483648.0f;
    *ry = (float)(zy & 0x7fffffffu) / 2147483648.0f;
}

}  // namespace

extern "C" {

// Per-frame inputs: the uniform buffer (pos, rst, lat) and the constants the shader bakes in.
struct OraclePtFrame {
    float pos[3], rst, lat[3], pad;
    uint32_t width, height;
    float aspect, sinfov, powc, pad2;
};

// sin and cos as the bounce computes them (for the accuracy test).
void oracle_pt_sincos(const float *theta, uint32_t n, float *s, float *c) {
    for (uint32_t i = 0; i < n; ++i) pt_sincos(theta[i], s + i, c + i);
}

// One sample() call: state_in and state_out hold four planes of width x height float4 each
// (o, d, t, b; pixel (x, y) at y * width + x).  state_in is not read when frame->rst != 0.
void oracle_pt_step(const uint32_t *nodes, const float *tris, uint32_t n, const float *state_in,
                    float *state_out, const OraclePtFrame *frame) {
    const uint32_t W = frame->width, H = frame->height;
    const size_t plane = (size_t)W * H * 4;
    const float sw_x = (float)W, sw_y = (float)H;
    const V3 pos = {frame->pos[0], frame->pos[1], frame->pos[2]};
    const V3 lat = {frame->lat[0], frame->lat[1], frame->lat[2]};
    const float eps = 0.0001f, two_pi = 0x1.921fb6p+2f;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t px = 0; px < (int64_t)W * H; ++px) {
        const uint32_t cx = (uint32_t)(px % W), cy = (uint32_t)(px / W);
        float o4[4] = {0, 0, 0, 0}, d4[4] = {0, 0, 0, 0}, t4[4] = {0, 0, 0, 0}, b4[4] = {0, 0, 0, 0};
        if (frame->rst == 0.0f) {
            std::memcpy(o4, state_in + 4 * px, 16);
            std::memcpy(d4, state_in + plane + 4 * px, 16);
            std::memcpy(t4, state_in + 2 * plane + 4 * px, 16);
            std::memcpy(b4, state_in + 3 * plane + 4 * px, 16);
        }
        // ptStep (:655-713)
        V3 o = {o4[0], o4[1], o4[2]}, d = {d4[0], d4[1], d4[2]}, b = {b4[0], b4[1], b4[2]};
        float seed = o4[3], bounces = d4[3];
        const bool new_path = b.x == 0.0f && b.y == 0.0f && b.z == 0.0f;
        const bool frame0 = new_path && t4[3] == 0.0f;
        if (frame0) seed = (float)base_hash(cx, cy) / 4294967296.0f + 0.008f;
        if (new_path) {
            // getCameraRay(vec2f(coord) + rand2(seed), ...) (:720-734)
            float rx, ry;
            rand2(seed, &rx, &ry);
            float sx = ((float)cx + rx) / sw_x, sy = ((float)cy + ry) / sw_y;
            sx = sx * 2.0f - 1.0f;
            sy = sy * 2.0f - 1.0f;
            sy = -sy;
            const V3 local = {frame->aspect * sx * frame->sinfov, 1.0f, sy * frame->sinfov};
            const V3 forward = normalize(sub(lat, pos));
            const V3 right = normalize(V3{forward.y, -forward.x, 0.0f});
            const V3 up = cross(right, forward);
            o = pos;
            d = to_world(right, forward, up, normalize(local));
            seed += 2.0f;
            b = {1.0f, 1.0f, 1.0f};
        }
        float dist;
        const int32_t prim = oracle_trace_one(nodes, tris, n, &o.x, &d.x, &dist, nullptr);
        if (dist >= 0.0f) {
            // the hit triangle's normal, facing the (nudged) ray (:571-577, :616-617)
            const float *tr = tris + 12 * (size_t)prim;
            const V3 v0 = {tr[0], tr[1], tr[2]}, v1 = {tr[4], tr[5], tr[6]}, v2 = {tr[8], tr[9], tr[10]};
            V3 norm = normalize(cross(sub(v1, v0), sub(v2, v0)));
            V3 dn = d;
            dn.x = dn.x + (std::fabs(dn.x) < 1e-5f ? 1.0f : 0.0f) * 1e-5f;
            dn.y = dn.y + (std::fabs(dn.y) < 1e-5f ? 1.0f : 0.0f) * 1e-5f;
            dn.z = dn.z + (std::fabs(dn.z) < 1e-5f ? 1.0f : 0.0f) * 1e-5f;
            if (!(dot(dn, V3{-norm.x, -norm.y, -norm.z}) > 0.0f)) norm = {-norm.x, -norm.y, -norm.z};
            const V3 o1 = normalize(ortho(norm));
            const V3 o2 = normalize(cross(o1, norm));
            o = add(o, mul(d, dist));
            // lambertDiffuse: wi = cosineSampleHemisphere(rand2(seed)), c = pow(.3, 2.2)
            float r2x, r2y;
            rand2(seed, &r2x, &r2y);
            const float rr = std::sqrt(r2x > 0.0f ? r2x : 0.0f);
            float sn, cs;
            pt_sincos(two_pi * r2y, &sn, &cs);
            const float dx = rr * cs, dy = rr * sn;
            const float zz = 1.0f - dx * dx - dy * dy;
            const V3 wi = {dx, dy, std::sqrt(zz > 0.0f ? zz : 0.0f)};
            seed += 2.0f;
            b = {b.x * frame->powc, b.y * frame->powc, b.z * frame->powc};
            o = add(o, mul(mul(norm, 1.01f), eps));
            d = to_world(o1, o2, norm, wi);
            if (bounces > 3.0f) {
                const float q1 = 1.0f - b.y, q = 0.05f > q1 ? 0.05f : q1;
                float ux, uy;
                rand2(seed, &ux, &uy);
                if (ux < q) {
                    b = {0.0f, 0.0f, 0.0f};
                } else {
                    const float keep = 1.0f - q;
                    b = {b.x / keep, b.y / keep, b.z / keep};
                }
                seed += 2.0f;
            }
            if (b.x == 0.0f && b.y == 0.0f && b.z == 0.0f) {
                t4[0] = t4[0] + 0.0f;
                t4[1] = t4[1] + 0.0f;
                t4[2] = t4[2] + 0.0f;
                t4[3] = t4[3] + 1.0f;
                bounces = -1.0f;
            }
        } else {
            t4[0] = t4[0] + b.x * 8.0f;
            t4[1] = t4[1] + b.y * 8.0f;
            t4[2] = t4[2] + b.z * 8.0f;
            t4[3] = t4[3] + 1.0f;
            bounces = -1.0f;
            b = {0.0f, 0.0f, 0.0f};
        }
        const float oo[4] = {o.x, o.y, o.z, seed}, dd[4] = {d.x, d.y, d.z, bounces + 1.0f},
                    bb[4] = {b.x, b.y, b.z, 1.0f};
        std::memcpy(state_out + 4 * px, oo, 16);
        std::memcpy(state_out + plane + 4 * px, dd, 16);
        std::memcpy(state_out + 2 * plane + 4 * px, t4, 16);
        std::memcpy(state_out + 3 * plane + 4 * px, bb, 16);
    }
}

}  // extern "C"
