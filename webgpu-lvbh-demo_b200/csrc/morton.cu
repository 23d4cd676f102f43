// morton.cu - K1a scene-box reduction and K1b Morton keys (sm_100a).
//
// Restates compute_aabb_z_idx (scripts/bvh/kernels/aabb-z-idx.js:177-209) and, for the box,
// the host-side min/max of parse-obj.js:27-53.  Both kernels stream the 48-byte triangle soup
// once with 16-byte loads: a warp reads 32 triangles as 96 consecutive float4 (three fully
// coalesced 512-byte loads), transposes them through 1.5 KB of shared memory, and each lane
// then owns one triangle.  HBM-bound: 48 B read per triangle (+4 B key written by K1b).
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ void warp_minmax(float (&mn)[3], float (&mx)[3]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xFFFFFFFFu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xFFFFFFFFu, mx[a], o));
        }
    }
}

// K1a: min / max of every vertex coordinate.  Vertices are the float4 of the soup; the pad
// word is ignored.  fminf/fmaxf skip NaN (K1b reports non-finite input separately).
__global__ void __launch_bounds__(kThreads) k_bounds(const float4 *__restrict__ v, uint64_t nv,
                                                     Control *__restrict__ ctl) {
    float mn[3] = {INFINITY, INFINITY, INFINITY};
    float mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    const uint64_t stride = (uint64_t)gridDim.x * kThreads;
    uint64_t i = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    for (; i + 3 * stride < nv; i += 4 * stride) {
        float4 p[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) p[u] = ld_stream(v + i + u * stride);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            mn[0] = fminf(mn[0], p[u].x); mx[0] = fmaxf(mx[0], p[u].x);
            mn[1] = fminf(mn[1], p[u].y); mx[1] = fmaxf(mx[1], p[u].y);
            mn[2] = fminf(mn[2], p[u].z); mx[2] = fmaxf(mx[2], p[u].z);
        }
    }
    for (; i < nv; i += stride) {
        const float4 p = ld_stream(v + i);
        mn[0] = fminf(mn[0], p.x); mx[0] = fmaxf(mx[0], p.x);
        mn[1] = fminf(mn[1], p.y); mx[1] = fmaxf(mx[1], p.y);
        mn[2] = fminf(mn[2], p.z); mx[2] = fmaxf(mx[2], p.z);
    }
    warp_minmax(mn, mx);
    __shared__ float s[kWarps][6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) { s[warp][a] = mn[a]; s[warp][3 + a] = mx[a]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        float r = s[0][a];
        for (int w = 1; w < kWarps; ++w) r = a < 3 ? fminf(r, s[w][a]) : fmaxf(r, s[w][a]);
        if (a < 3) atomicMax(&ctl->bounds_ord[a], ~ord_lo(r));
        else atomicMax(&ctl->bounds_ord[a], ord_lo(r));
    }
}

// K1a for a soup whose box is reduced on the device: the box and every triangle's centroid in
// one read of triangles [t0, t1).  A warp loads a row of 32 triangles as three coalesced
// 512-byte loads (its next row in flight meanwhile), transposes it through shared memory so
// that each lane owns one triangle, and stores the centroids (box.max + box.min) * .5 in
// structure-of-arrays form (three coalesced 128-byte stores); K1b then reads 12 bytes per
// triangle instead of the soup's 48.  Box mins and maxes feed the scene box (fminf / fmaxf are
// exact, so the box is the min / max over every vertex whatever the order); non-finite
// vertices set ERR_NONFINITE.  Launched per chunk of the soup, it can run behind the chunk's
// upload.
__global__ void __launch_bounds__(kThreads) k_bounds_cen(const float4 *__restrict__ tri, uint32_t t0, uint32_t t1,
                                                         float *__restrict__ cen, uint32_t stride,
                                                         Control *__restrict__ ctl) {
    __shared__ float4 stage[kWarps][96];
    __shared__ float s[kWarps][6];
    float mn[3] = {INFINITY, INFINITY, INFINITY};
    float mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rows = (t1 - t0 + 31u) / 32u;
    const uint32_t nw = gridDim.x * kWarps;
    const uint64_t nv = 3ull * t1;
    bool bad = false;
    float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = q0, q2 = q0;
    auto ld_row = [&](uint32_t r) {
        const uint64_t base = 3ull * (t0 + 32ull * r);
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        q0 = base + lane < nv ? ld_stream(tri + base + lane) : z;
        q1 = base + 32 + lane < nv ? ld_stream(tri + base + 32 + lane) : z;
        q2 = base + 64 + lane < nv ? ld_stream(tri + base + 64 + lane) : z;
    };
    uint32_t r = blockIdx.x * kWarps + warp;
    if (r < rows) ld_row(r);
    for (; r < rows; r += nw) {
        const float4 a0 = q0, a1 = q1, a2 = q2;
        if (r + nw < rows) ld_row(r + nw);
        stage[warp][lane] = a0;
        stage[warp][32 + lane] = a1;
        stage[warp][64 + lane] = a2;
        __syncwarp();
        const float4 v0 = stage[warp][3 * lane], v1 = stage[warp][3 * lane + 1], v2 = stage[warp][3 * lane + 2];
        __syncwarp();
        const uint32_t t = t0 + 32u * r + lane;
        if (t < t1) {
            bad |= !(finite3(v0) && finite3(v1) && finite3(v2));
            // box.min = min(v0, min(v1, v2)); box.max = max(v0, max(v1, v2))   (aabb-z-idx.js:186-187)
            const float nx = fminf(v0.x, fminf(v1.x, v2.x)), ny = fminf(v0.y, fminf(v1.y, v2.y)), nz = fminf(v0.z, fminf(v1.z, v2.z));
            const float xx = fmaxf(v0.x, fmaxf(v1.x, v2.x)), xy = fmaxf(v0.y, fmaxf(v1.y, v2.y)), xz = fmaxf(v0.z, fmaxf(v1.z, v2.z));
            __stcs(cen + t, centroid(nx, xx));
            __stcs(cen + stride + t, centroid(ny, xy));
            __stcs(cen + 2ull * stride + t, centroid(nz, xz));
            mn[0] = fminf(mn[0], nx); mn[1] = fminf(mn[1], ny); mn[2] = fminf(mn[2], nz);
            mx[0] = fmaxf(mx[0], xx); mx[1] = fmaxf(mx[1], xy); mx[2] = fmaxf(mx[2], xz);
        }
    }
    warp_minmax(mn, mx);
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) { s[warp][a] = mn[a]; s[warp][3 + a] = mx[a]; }
    }
    if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(&ctl->err, ERR_NONFINITE);
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        float v = s[0][a];
        for (int w = 1; w < kWarps; ++w) v = a < 3 ? fminf(v, s[w][a]) : fmaxf(v, s[w][a]);
        if (a < 3) atomicMax(&ctl->bounds_ord[a], ~ord_lo(v));
        else atomicMax(&ctl->bounds_ord[a], ord_lo(v));
    }
}

// K1b: per triangle box, centroid, quantisation and 30-bit Morton key, written in input order.
// One block per chunk of sort_chunk_tiles(n) sort tiles: per tile each warp takes chunks of 32
// triangles (96 consecutive float4, three coalesced 512-byte loads, transposed through shared
// memory so that each lane owns a triangle); the digit counts of all three sort passes
// accumulate over the block, and the counts of the first pass's digit per tile and per chunk
// go straight to the sort's scratch, so the first sort pass starts from them.
// kSrcMesh: the triangles are index triples into a buffer of 16-byte vertex rows (the indexed
// leaf format's input); each lane gathers its triangle's three rows, an index past the buffer
// reads row 0 and sets ERR_BAD_INDEX.  The centroids K1a stored are quantised by k_morton_cen.
constexpr int kSrcSoup = 0, kSrcMesh = 1;
template <int SRC, int THREADS = kThreads>
__global__ void __launch_bounds__(THREADS) k_morton(const float4 *__restrict__ tri, uint32_t n,
                                                     HostBounds hb, Control *__restrict__ ctl,
                                                     uint32_t *__restrict__ keys,
                                                     uint32_t *__restrict__ epoch, uint32_t chunk_tiles,
                                                     uint32_t *__restrict__ tile_hist,
                                                     uint32_t *__restrict__ chunk_sum,
                                                     const uint32_t *__restrict__ idx3, uint32_t nverts,
                                                     uint32_t chunk0) {
    constexpr bool MESH = SRC == kSrcMesh;
    const uint32_t chunk = chunk0 + blockIdx.x;  // this block's chunk of sort tiles
    constexpr int P = kDigits / THREADS;  // digits per thread in the per-tile counts
    constexpr int WARPS = THREADS / 32;
    __shared__ float4 stage[MESH ? 1 : WARPS][96];
    __shared__ uint32_t th[kDigits];
    if (chunk == 0 && threadIdx.x == 0) {  // new arrival epoch for K3c; 0 is never used
        const uint32_t e = *epoch + 1u;
        *epoch = e == 0u ? 1u : e;
    }

    float umin[3], umax[3];
    if (hb.use) {
#pragma unroll
        for (int a = 0; a < 3; ++a) { umin[a] = hb.v[a]; umax[a] = hb.v[3 + a]; }
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            umin[a] = ord_lo_inv(~ctl->bounds_ord[a]);
            umax[a] = ord_lo_inv(ctl->bounds_ord[3 + a]);
        }
    }

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t nv = 3ull * n;
    const uint32_t tiles = sort_tiles(n);
    uint32_t acc[P];
#pragma unroll
    for (int j = 0; j < P; ++j) acc[j] = 0;
    bool bad = false, bad_index = false;
    for (uint32_t tt = 0; tt < chunk_tiles; ++tt) {
        const uint32_t tile = chunk * chunk_tiles + tt;
        if (tile >= tiles) break;  // uniform across the block
        for (int i = threadIdx.x; i < kDigits; i += THREADS) th[i] = 0;
        __syncthreads();
        bool coherent = false;
        // soup: a warp's next row of 32 triangles (three coalesced float4 per lane) is loaded
        // while it works on this one (0.179 -> 0.157 ms on 16.7 M triangles)
        float4 q0 = make_float4(0.f, 0.f, 0.f, 0.f), q1 = q0, q2 = q0;
        auto ld_row = [&](uint32_t cc) {
            const uint64_t base = 3ull * (tile * (uint32_t)kSortTile + 32u * cc);
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            q0 = base + lane < nv ? ld_stream(tri + base + lane) : z;
            q1 = base + 32 + lane < nv ? ld_stream(tri + base + 32 + lane) : z;
            q2 = base + 64 + lane < nv ? ld_stream(tri + base + 64 + lane) : z;
        };
        if (!MESH && tile * (uint32_t)kSortTile + 32u * warp < n) ld_row(warp);
        for (uint32_t c = warp; c < (uint32_t)kSortTile / 32; c += WARPS) {
            const uint32_t t0 = tile * (uint32_t)kSortTile + 32u * c;
            if (t0 >= n) break;
            const uint32_t t = t0 + lane;
            const bool valid = t < n;
            float4 v0, v1, v2;
            if constexpr (MESH) {
                uint32_t i0 = 0, i1 = 0, i2 = 0;
                if (valid) {
                    i0 = __ldcs(idx3 + 3ull * t);
                    i1 = __ldcs(idx3 + 3ull * t + 1);
                    i2 = __ldcs(idx3 + 3ull * t + 2);
                    if (i0 >= nverts || i1 >= nverts || i2 >= nverts) {
                        bad_index = true;
                        i0 = i0 < nverts ? i0 : 0u;
                        i1 = i1 < nverts ? i1 : 0u;
                        i2 = i2 < nverts ? i2 : 0u;
                    }
                }
                v0 = __ldg(tri + i0);
                v1 = __ldg(tri + i1);
                v2 = __ldg(tri + i2);
            } else {
                const float4 a0 = q0, a1 = q1, a2 = q2;
                if (c + WARPS < (uint32_t)kSortTile / 32 && t0 + 32u * WARPS < n) ld_row(c + WARPS);
                stage[warp][lane] = a0;
                stage[warp][32 + lane] = a1;
                stage[warp][64 + lane] = a2;
                __syncwarp();
                v0 = stage[warp][3 * lane];
                v1 = stage[warp][3 * lane + 1];
                v2 = stage[warp][3 * lane + 2];
                __syncwarp();
            }
            uint32_t key = 0;
            if (valid) {
                bad |= !(finite3(v0) && finite3(v1) && finite3(v2));
                // box.min = min(v0, min(v1, v2)); box.max = max(v0, max(v1, v2))   (:186-187)
                const uint32_t qx = quantise(fminf(v0.x, fminf(v1.x, v2.x)), fmaxf(v0.x, fmaxf(v1.x, v2.x)), umin[0], umax[0]);
                const uint32_t qy = quantise(fminf(v0.y, fminf(v1.y, v2.y)), fmaxf(v0.y, fmaxf(v1.y, v2.y)), umin[1], umax[1]);
                const uint32_t qz = quantise(fminf(v0.z, fminf(v1.z, v2.z)), fmaxf(v0.z, fmaxf(v1.z, v2.z)), umin[2], umax[2]);
                key = morton3(qx, qy, qz);
                keys[t] = key;
            }
            // repeated digits over consecutive lanes (coherent input) are counted once per run;
            // the warp tests its first chunk of each tile and keeps the answer for the tile
            if (c == (uint32_t)warp) coherent = runs_few(key & (kDigits - 1), valid);
            if (coherent) add_runs(th, key & (kDigits - 1), valid);
            else if (valid) atomicAdd(&th[key & (kDigits - 1)], 1u);
        }
        __syncthreads();
        uint32_t *row = tile_hist + (size_t)tile * kDigits + threadIdx.x * P;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const uint32_t c = th[threadIdx.x * P + j];
            row[j] = c;
            acc[j] += c;
        }
        __syncthreads();
    }
    // the chunk's counts, and its share of the pass's global digit counts (one of the partial
    // rows; the later passes' counts come from their own tile-histogram pass)
    uint32_t *crow = chunk_sum + (size_t)chunk * kDigits + threadIdx.x * P;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        crow[j] = acc[j];
        if (acc[j]) atomicAdd(&ctl->hist_part[0][chunk % kHistParts][threadIdx.x * P + j], acc[j]);
    }
    if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(&ctl->err, ERR_NONFINITE);
    if (__any_sync(0xFFFFFFFFu, bad_index) && lane == 0) atomicOr(&ctl->err, ERR_BAD_INDEX);
}

// K1b from the centroids K1a stored (structure of arrays, `cen_stride` floats apart, a multiple
// of 4): one block per chunk of sort tiles, each tile's three 16 KB centroid runs copied into
// shared memory by 16-byte cp.async while the block quantises the tile before (two buffers), so
// that a whole tile's loads are in flight at once.  Row i of warp w is keys 32 (w + WARPS i) ..
// + 31 of the tile, one per lane; counts as k_morton.  On 16.7 M clustered centroids (B200):
// 0.104 ms as k_morton's centroid mode (a warp's next row of 32 loaded while it works on this
// one: about 12 KB in flight per SM), 0.091 ms so with 512 threads, 0.087 ms with 1024.  The
// division of quantise_cen is not what bounds it: taking it out of the common case (a product
// with a per-axis reciprocal, exact except within 2^-11 of a step, those keys divided) was
// slower (0.089 -> 0.100 ms at 512 threads), though exact over every float.
constexpr int kCenThreads = 1024;
struct CenSmem {
    float c[2][3][kSortTile];  // [buffer][axis][key of the tile]
};
__global__ void __launch_bounds__(kCenThreads) k_morton_cen(const float *__restrict__ cen, uint32_t cen_stride,
                                                            uint32_t n, Control *__restrict__ ctl,
                                                            uint32_t *__restrict__ keys, uint32_t *__restrict__ epoch,
                                                            uint32_t chunk_tiles, uint32_t *__restrict__ tile_hist,
                                                            uint32_t *__restrict__ chunk_sum) {
    constexpr int WARPS = kCenThreads / 32, P = kDigits / kCenThreads, R = kSortTile / 32 / WARPS;
    static_assert(R * WARPS * 32 == kSortTile && P * kCenThreads == kDigits, "whole rows and digits");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CenSmem &S = *reinterpret_cast<CenSmem *>(smem_raw);
    __shared__ uint32_t th[2][kDigits];  // a tile's counts, alternating with the buffers
    const uint32_t chunk = blockIdx.x;
    chain_wait();
    if (chunk == 0 && threadIdx.x == 0) {  // new arrival epoch for K3c; 0 is never used
        const uint32_t e = *epoch + 1u;
        *epoch = e == 0u ? 1u : e;
    }
    float umin[3], umax[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        umin[a] = ord_lo_inv(~ctl->bounds_ord[a]);
        umax[a] = ord_lo_inv(ctl->bounds_ord[3 + a]);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tiles = sort_tiles(n), t0 = chunk * chunk_tiles, t1 = min(tiles, t0 + chunk_tiles);
    // a tile's 16-byte pieces of the three runs up to the one holding key n - 1 (the stride
    // keeps every run on a 16-byte boundary; a partial last piece reads stride slack)
    auto issue = [&](uint32_t tile, int b) {
        const uint32_t first = tile * (uint32_t)kSortTile;
        const uint32_t pieces = min((uint32_t)kSortTile, n - first + 3u) / 4u;
        for (uint32_t q = threadIdx.x; q < 3u * (kSortTile / 4); q += kCenThreads) {
            const uint32_t a = q / (kSortTile / 4), p = q % (kSortTile / 4);
            if (p < pieces) cp_async16(&S.c[b][a][4 * p], cen + (size_t)a * cen_stride + first + 4 * p);
        }
        cp_async_commit();
    };
    uint32_t acc[P];
#pragma unroll
    for (int j = 0; j < P; ++j) acc[j] = 0;
    if (t0 < t1) issue(t0, 0);
    for (uint32_t tile = t0; tile < t1; ++tile) {
        const int b = (int)((tile - t0) & 1u);
        if (tile + 1 < t1) issue(tile + 1, b ^ 1);
        else cp_async_commit();  // an empty group keeps the count below uniform
        for (int i = threadIdx.x; i < kDigits; i += kCenThreads) th[b][i] = 0;
        asm volatile("cp.async.wait_group 1;" ::: "memory");  // this tile's pieces (own ones)
        __syncthreads();  // everyone's pieces, and the cleared counts
        bool coherent = false;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int j = 32 * (warp + WARPS * i) + lane;
            const uint32_t t = tile * (uint32_t)kSortTile + j;
            const bool valid = t < n;
            uint32_t key = 0;
            if (valid) {
                key = morton3(quantise_cen(S.c[b][0][j], umin[0], umax[0]), quantise_cen(S.c[b][1][j], umin[1], umax[1]),
                              quantise_cen(S.c[b][2][j], umin[2], umax[2]));
                keys[t] = key;
            }
            // repeated digits over consecutive lanes (coherent input) are counted once per run;
            // the warp tests its first row of each tile and keeps the answer for the tile
            if (i == 0) coherent = runs_few(key & (kDigits - 1), valid);
            if (coherent) add_runs(th[b], key & (kDigits - 1), valid);
            else if (valid) atomicAdd(&th[b][key & (kDigits - 1)], 1u);
        }
        __syncthreads();  // the tile's counts are complete; buffer b is read
        uint32_t *row = tile_hist + (size_t)tile * kDigits + threadIdx.x * P;
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const uint32_t c = th[b][threadIdx.x * P + j];
            row[j] = c;
            acc[j] += c;
        }
        // no barrier here: the next tile counts into th[b ^ 1], which this tile's first barrier
        // found read, and refills buffer b ^ 1 only, read before this tile's second barrier
    }
    uint32_t *crow = chunk_sum + (size_t)chunk * kDigits + threadIdx.x * P;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        crow[j] = acc[j];
        if (acc[j]) atomicAdd(&ctl->hist_part[0][chunk % kHistParts][threadIdx.x * P + j], acc[j]);
    }
}

// K1a for a mesh: min / max over the vertices the triangles use (the rows of unused vertices
// take no part, as in the soup), three gathers of 16-byte rows per triangle.  Indices past the
// buffer are skipped (K1b reports them).
__global__ void __launch_bounds__(kThreads) k_bounds_mesh(const float4 *__restrict__ verts, uint32_t nverts,
                                                          const uint32_t *__restrict__ idx3, uint32_t n,
                                                          Control *__restrict__ ctl) {
    float mn[3] = {INFINITY, INFINITY, INFINITY};
    float mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    const uint32_t stride = gridDim.x * kThreads;
    for (uint64_t e = (uint64_t)blockIdx.x * kThreads + threadIdx.x; e < 3ull * n; e += stride) {
        const uint32_t vi = __ldcs(idx3 + e);
        if (vi >= nverts) continue;
        const float4 p = __ldg(verts + vi);
        mn[0] = fminf(mn[0], p.x); mx[0] = fmaxf(mx[0], p.x);
        mn[1] = fminf(mn[1], p.y); mx[1] = fmaxf(mx[1], p.y);
        mn[2] = fminf(mn[2], p.z); mx[2] = fmaxf(mx[2], p.z);
    }
    warp_minmax(mn, mx);
    __shared__ float s[kWarps][6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) { s[warp][a] = mn[a]; s[warp][3 + a] = mx[a]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        float r = s[0][a];
        for (int w = 1; w < kWarps; ++w) r = a < 3 ? fminf(r, s[w][a]) : fmaxf(r, s[w][a]);
        if (a < 3) atomicMax(&ctl->bounds_ord[a], ~ord_lo(r));
        else atomicMax(&ctl->bounds_ord[a], ord_lo(r));
    }
}

// The indexed leaf format's triangle rows: the three vertex indices of each sorted triangle.
__global__ void __launch_bounds__(256) k_leaf_idx(const uint32_t *__restrict__ idx3, const uint32_t *__restrict__ perm,
                                                  uint32_t n, uint32_t *__restrict__ sidx) {
    const uint32_t i = blockIdx.x * 256u + threadIdx.x;
    if (i >= n) return;
    uint32_t ti = __ldcs(perm + i);
    ti = ti < n ? ti : 0u;  // a permutation entry is below n
    const uint32_t *src = idx3 + 3ull * ti;
    const uint32_t a = __ldg(src), b = __ldg(src + 1), c = __ldg(src + 2);
    sidx[3ull * i] = a;
    sidx[3ull * i + 1] = b;
    sidx[3ull * i + 2] = c;
}

// Batched K1a: one block per sort tile (at most kSortTile triangles of one segment); the
// tile's vertex box goes into its segment's six ordered bound words.
__global__ void __launch_bounds__(kThreads) k_bounds_batch(const float4 *__restrict__ tri,
                                                           const SegRow *__restrict__ rows,
                                                           const uint32_t *__restrict__ tile_seg,
                                                           const float *__restrict__ host_bounds,
                                                           uint32_t *__restrict__ seg_ord) {
    const uint32_t tile = blockIdx.x, sg = __ldg(tile_seg + tile);
    if (host_bounds && !isnan(__ldg(host_bounds + 6ull * sg))) return;  // bounds given
    const uint32_t t0 = __ldg(&rows[sg].tri), t1 = __ldg(&rows[sg + 1].tri);
    const uint32_t first = t0 + (tile - __ldg(&rows[sg].tile)) * (uint32_t)kSortTile;
    const uint32_t cnt = min((uint32_t)kSortTile, t1 - first);
    const float4 *v = tri + 3ull * first;
    const uint32_t nv = 3u * cnt;
    float mn[3] = {INFINITY, INFINITY, INFINITY};
    float mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = threadIdx.x; i < nv; i += kThreads) {
        const float4 p = ld_stream(v + i);
        mn[0] = fminf(mn[0], p.x); mx[0] = fmaxf(mx[0], p.x);
        mn[1] = fminf(mn[1], p.y); mx[1] = fmaxf(mx[1], p.y);
        mn[2] = fminf(mn[2], p.z); mx[2] = fmaxf(mx[2], p.z);
    }
    warp_minmax(mn, mx);
    __shared__ float s[kWarps][6];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) { s[warp][a] = mn[a]; s[warp][3 + a] = mx[a]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        float r = s[0][a];
        for (int w = 1; w < kWarps; ++w) r = a < 3 ? fminf(r, s[w][a]) : fmaxf(r, s[w][a]);
        uint32_t *o = seg_ord + 6ull * sg;
        if (a < 3) atomicMax(o + a, ~ord_lo(r));
        else atomicMax(o + a, ord_lo(r));
    }
}

// Batched K1b: one block per sort tile; each warp takes chunks of 32 triangles of the tile
// (the same transposed 16-byte loads as k_morton), quantises them with the segment's bounds
// and adds the tile's digit counts to the segment's histograms.
template <int BITS>
__global__ void __launch_bounds__(kThreads) k_morton_batch(const float4 *__restrict__ tri,
                                                           const SegRow *__restrict__ rows,
                                                           const uint32_t *__restrict__ tile_seg,
                                                           const float *__restrict__ host_bounds,
                                                           const uint32_t *__restrict__ seg_ord,
                                                           uint32_t *__restrict__ seg_hist,
                                                           Control *__restrict__ ctl,
                                                           uint32_t *__restrict__ keys,
                                                           uint32_t *__restrict__ epoch) {
    constexpr int D = 1 << BITS, NP = BITS == kDigitBits ? kSortPasses : kSortPasses32;
    static_assert(NP * D <= kHistWords, "per-segment counts");
    __shared__ float4 stage[kWarps][96];
    __shared__ uint32_t hist[NP][D];
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // new arrival epoch for K3c; 0 is never used
        const uint32_t e = *epoch + 1u;
        *epoch = e == 0u ? 1u : e;
    }
    for (int i = threadIdx.x; i < NP * D; i += kThreads) (&hist[0][0])[i] = 0;
    const uint32_t tile = blockIdx.x, sg = __ldg(tile_seg + tile);
    const uint32_t t0 = __ldg(&rows[sg].tri), t1 = __ldg(&rows[sg + 1].tri);
    const uint32_t first = t0 + (tile - __ldg(&rows[sg].tile)) * (uint32_t)kSortTile;
    const uint32_t cnt = min((uint32_t)kSortTile, t1 - first);
    float umin[3], umax[3];
    if (host_bounds && !isnan(host_bounds[6ull * sg])) {
#pragma unroll
        for (int a = 0; a < 3; ++a) { umin[a] = host_bounds[6ull * sg + a]; umax[a] = host_bounds[6ull * sg + 3 + a]; }
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            umin[a] = ord_lo_inv(~seg_ord[6ull * sg + a]);
            umax[a] = ord_lo_inv(seg_ord[6ull * sg + 3 + a]);
        }
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float4 *src = tri + 3ull * first;
    const uint32_t nv = 3u * cnt;
    bool bad = false, coherent = false;
    const uint32_t rows_n = (cnt + 31) / 32;
    // a warp's next row of 32 triangles is loaded while it works on this one
    float4 q[3];
    auto ld_row = [&](uint32_t cc) {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const uint32_t e = 96u * cc + 32 * r + lane;
            q[r] = e < nv ? ld_stream(src + e) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    if ((uint32_t)warp < rows_n) ld_row(warp);
    for (uint32_t c = warp; c < rows_n; c += kWarps) {
        const float4 a0 = q[0], a1 = q[1], a2 = q[2];
        if (c + kWarps < rows_n) ld_row(c + kWarps);
        stage[warp][lane] = a0;
        stage[warp][32 + lane] = a1;
        stage[warp][64 + lane] = a2;
        __syncwarp();
        const float4 v0 = stage[warp][3 * lane], v1 = stage[warp][3 * lane + 1],
                     v2 = stage[warp][3 * lane + 2];
        __syncwarp();
        const uint32_t t = 32u * c + lane;
        const bool valid = t < cnt;
        uint32_t key = 0;
        if (valid) {
            bad |= !(finite3(v0) && finite3(v1) && finite3(v2));
            const uint32_t qx = quantise(fminf(v0.x, fminf(v1.x, v2.x)), fmaxf(v0.x, fmaxf(v1.x, v2.x)), umin[0], umax[0]);
            const uint32_t qy = quantise(fminf(v0.y, fminf(v1.y, v2.y)), fmaxf(v0.y, fmaxf(v1.y, v2.y)), umin[1], umax[1]);
            const uint32_t qz = quantise(fminf(v0.z, fminf(v1.z, v2.z)), fmaxf(v0.z, fmaxf(v1.z, v2.z)), umin[2], umax[2]);
            key = morton3(qx, qy, qz);
            keys[first + t] = key;
        }
        if (c == (uint32_t)warp) coherent = runs_few(key >> (BITS * (NP - 1)), valid);
        if (coherent) {
#pragma unroll
            for (int p = 0; p < NP; ++p) add_runs(hist[p], (key >> (BITS * p)) & (D - 1), valid);
        } else if (valid) {
#pragma unroll
            for (int p = 0; p < NP; ++p) atomicAdd(&hist[p][(key >> (BITS * p)) & (D - 1)], 1u);
        }
    }
    if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(&ctl->err, ERR_NONFINITE);
    __syncthreads();
    uint32_t *h = seg_hist + (size_t)sg * kHistWords;
    for (int i = threadIdx.x; i < NP * D; i += kThreads) {
        const uint32_t c = (&hist[0][0])[i];
        if (c) atomicAdd(h + i, c);
    }
}

// Segment of every sort tile and tree block: one warp per segment fills its entries.
__global__ void __launch_bounds__(256) k_seg_tables(const SegRow *__restrict__ rows, uint32_t num_segs,
                                                    uint32_t *__restrict__ tile_seg,
                                                    uint32_t *__restrict__ blk_seg,
                                                    uint32_t *__restrict__ grp_seg) {
    const uint32_t sg = (blockIdx.x * 256u + threadIdx.x) / 32u, lane = threadIdx.x & 31;
    if (sg >= num_segs) return;
    const SegRow a = rows[sg], b = rows[sg + 1];
    for (uint32_t t = a.tile + lane; t < b.tile; t += 32) tile_seg[t] = sg;
    for (uint32_t t = a.blk + lane; t < b.blk; t += 32) blk_seg[t] = sg;
    for (uint32_t t = a.grp + lane; t < b.grp; t += 32) grp_seg[t] = sg;
}

__global__ void k_gather_indexed(const float *__restrict__ xyz, uint32_t num_verts,
                                 const uint32_t *__restrict__ idx3, uint32_t n,
                                 float4 *__restrict__ tri, uint32_t *__restrict__ err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const uint32_t vi = __ldg(idx3 + 3ull * t + v);
        if (vi >= num_verts) {
            atomicOr(err, ERR_BAD_INDEX);
            tri[3ull * t + v] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const float *p = xyz + 3ull * vi;
        tri[3ull * t + v] = make_float4(__ldg(p), __ldg(p + 1), __ldg(p + 2), 0.0f);
    }
}

}  // namespace

void launch_bounds(const float4 *tri, uint32_t n, Control *ctl, cudaStream_t s) {
    const uint64_t nv = 3ull * n;
    uint64_t blocks = (nv + kThreads * 4 - 1) / (kThreads * 4);
    const uint64_t cap = (uint64_t)sm_count() * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_bounds<<<(unsigned)blocks, kThreads, 0, s>>>(tri, nv, ctl);
}

void launch_morton(const float4 *tri, uint32_t n, HostBounds hb, Control *ctl, uint32_t *keys,
                   uint32_t *epoch, uint32_t *sort_scratch, cudaStream_t s) {
    if (n == 0) return;
    launch_morton_chunks(tri, n, hb, ctl, keys, epoch, sort_scratch, 0, sort_chunks(n), s);
}

void launch_morton_chunks(const float4 *tri, uint32_t n, HostBounds hb, Control *ctl, uint32_t *keys,
                          uint32_t *epoch, uint32_t *sort_scratch, uint32_t c0, uint32_t c1, cudaStream_t s) {
    if (n == 0 || c1 <= c0) return;
    k_morton<kSrcSoup><<<c1 - c0, kThreads, 0, s>>>(tri, n, hb, ctl, keys, epoch, sort_chunk_tiles(n),
                                                    sort_scratch, sort_chunk_sums(sort_scratch, n), nullptr, 0u,
                                                    c0);
}

void launch_bounds_cen(const float4 *tri, uint32_t t0, uint32_t t1, float *cen, uint32_t cen_stride,
                       Control *ctl, cudaStream_t s) {
    if (t1 <= t0) return;
    uint32_t blocks = (t1 - t0 + 32u * kWarps - 1) / (32u * kWarps);
    const uint32_t cap = (uint32_t)sm_count() * 8u;
    if (blocks > cap) blocks = cap;
    k_bounds_cen<<<blocks, kThreads, 0, s>>>(tri, t0, t1, cen, cen_stride, ctl);
}

void launch_morton_cen(const float *cen, uint32_t cen_stride, uint32_t n, Control *ctl, uint32_t *keys,
                       uint32_t *epoch, uint32_t *sort_scratch, cudaStream_t s) {
    if (n == 0) return;
    launch_chained(chain_build(n), k_morton_cen, sort_chunks(n), kCenThreads, sizeof(CenSmem), s, cen, cen_stride, n, ctl, keys,
                   epoch, sort_chunk_tiles(n), sort_scratch, sort_chunk_sums(sort_scratch, n));
}

cudaError_t morton_init() {
    return cudaFuncSetAttribute(k_morton_cen, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(CenSmem));
}

void launch_bounds_mesh(const float4 *verts, uint32_t nverts, const uint32_t *idx3, uint32_t n, Control *ctl,
                        cudaStream_t s) {
    uint64_t blocks = (3ull * n + kThreads * 4 - 1) / (kThreads * 4);
    const uint64_t cap = (uint64_t)sm_count() * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_bounds_mesh<<<(unsigned)blocks, kThreads, 0, s>>>(verts, nverts, idx3, n, ctl);
}

void launch_morton_mesh(const float4 *verts, uint32_t nverts, const uint32_t *idx3, uint32_t n, HostBounds hb,
                        Control *ctl, uint32_t *keys, uint32_t *epoch, uint32_t *sort_scratch, cudaStream_t s) {
    if (n == 0) return;
    k_morton<kSrcMesh><<<sort_chunks(n), kThreads, 0, s>>>(verts, n, hb, ctl, keys, epoch, sort_chunk_tiles(n),
                                                           sort_scratch, sort_chunk_sums(sort_scratch, n), idx3,
                                                           nverts, 0u);
}

void launch_leaf_idx(const uint32_t *idx3, const uint32_t *perm, uint32_t n, uint32_t *sidx, cudaStream_t s) {
    if (n == 0) return;
    k_leaf_idx<<<(n + 255) / 256, 256, 0, s>>>(idx3, perm, n, sidx);
}

void launch_gather_indexed(const float *xyz, uint32_t num_verts, const uint32_t *idx3,
                           uint32_t n, float4 *tri, uint32_t *err, cudaStream_t s) {
    if (n == 0) return;
    k_gather_indexed<<<(n + 255) / 256, 256, 0, s>>>(xyz, num_verts, idx3, n, tri, err);
}

void launch_seg_tables(const SegRow *rows, uint32_t num_segs, uint32_t *tile_seg,
                       uint32_t *blk_seg, uint32_t *grp_seg, cudaStream_t s) {
    if (num_segs == 0) return;
    k_seg_tables<<<(num_segs + 7) / 8, 256, 0, s>>>(rows, num_segs, tile_seg, blk_seg, grp_seg);
}

void launch_bounds_batch(const BatchPlan &bp, const float4 *tri, const float *host_bounds,
                         uint32_t *seg_ord, cudaStream_t s) {
    if (bp.tiles == 0) return;
    k_bounds_batch<<<bp.tiles, kThreads, 0, s>>>(tri, bp.rows, bp.tile_seg, host_bounds, seg_ord);
}

void launch_morton_batch(const BatchPlan &bp, const float4 *tri, const float *host_bounds,
                         const uint32_t *seg_ord, uint32_t *seg_hist, Control *ctl,
                         uint32_t *keys_out, uint32_t *epoch, cudaStream_t s) {
    if (bp.tiles == 0) return;
    if (bp.digit_bits == kDigitBits32)
        k_morton_batch<kDigitBits32><<<bp.tiles, kThreads, 0, s>>>(tri, bp.rows, bp.tile_seg, host_bounds,
                                                                   seg_ord, seg_hist, ctl, keys_out, epoch);
    else
        k_morton_batch<kDigitBits><<<bp.tiles, kThreads, 0, s>>>(tri, bp.rows, bp.tile_seg, host_bounds,
                                                                 seg_ord, seg_hist, ctl, keys_out, epoch);
}

}  // namespace lvbh
