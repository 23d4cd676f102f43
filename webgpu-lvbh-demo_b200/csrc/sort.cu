// sort.cu - K2: onesweep stable LSD radix sort pass of (Morton key, triangle index) (sm_100a).
//
// Replaces the reference's 2-bit x 16-pass sort (scripts/bvh/kernels/radix-sort.js:162-499:
// init_idx, init_off, two scan_up levels and scan_and_sort per pass, 64 submits and 16 host
// waits).  Its result is the stable argsort of the keys - ties keep ascending input index -
// and this pass keeps that contract with 8-bit digits, four passes over 32 bits:
//
//   * the global digit counts of every pass come from K1b's histograms (one read of the keys);
//   * a tile of 4096 keys (256 threads x 16) is ranked in shared memory: each warp walks its
//     keys in input order, __match_any_sync groups equal digits, and the peers' lane order
//     plus a per-warp running count gives each key its stable rank;
//   * the tile's digit counts are combined with earlier tiles by decoupled look-back: tiles
//     are numbered by an atomic counter in launch order, each publishes its counts (flag
//     AGGREGATE) and then its inclusive prefix (flag PREFIX) in one 32-bit word per digit, and
//     looks back only at tiles that have already started, so the waits always end;
//   * every wait is bounded (kSpinLimitCycles); past it the kernel records ERR_LOOKBACK_TIMEOUT
//     and carries on, so it never hangs;
//   * keys and values are staged in digit order in shared memory and written out so that
//     consecutive threads write consecutive addresses of each digit's run.
//
// HBM-bound: per key one 4-byte key read (+4-byte value read after the first pass) and two
// 4-byte writes.
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

constexpr int T = kSortThreads;
constexpr int W = T / 32;
constexpr int IPT = kSortItems;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1u;
constexpr int kLookback = 8;  // predecessor tiles read per look-back step

static_assert(T == kDigits, "one thread per digit in the per-digit phases");

// Exclusive scan of one value per thread across the block; returns the thread's prefix.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t *s_warp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t warp_off = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) warp_off += (w < warp) ? s_warp[w] : 0u;
    __syncthreads();
    return warp_off + incl - x;
}

// The keys a tile works on: its segment's first key in the batch and size, the tile's first
// key within the segment, the segment's first tile (the look-back stops there) and the
// segment's digit counts for this pass.  The plain sort is the one-segment case.
struct TileSpan {
    size_t start;
    uint32_t n, base, first;
    const uint32_t *hist;
};

struct OneSegSort {
    uint32_t n;
    const uint32_t *hist;  // this pass's counts
    __device__ __forceinline__ TileSpan span(uint32_t tile) const {
        return TileSpan{0, n, tile * (uint32_t)kSortTile, 0u, hist};
    }
};

struct ManySegSort {
    const SegRow *rows;
    const uint32_t *tile_seg;
    const uint32_t *seg_hist;  // [segment][pass][digit]
    int pass;
    __device__ __forceinline__ TileSpan span(uint32_t tile) const {
        const uint32_t sg = __ldg(tile_seg + tile);
        const uint32_t t0 = __ldg(&rows[sg].tri), t1 = __ldg(&rows[sg + 1].tri);
        const uint32_t first = __ldg(&rows[sg].tile);
        return TileSpan{t0, t1 - t0, (tile - first) * (uint32_t)kSortTile, first,
                        seg_hist + ((size_t)sg * kSortPasses + pass) * kDigits};
    }
};

template <class Segs>
__global__ void __launch_bounds__(T, 4) k_onesweep(Segs segs, const uint32_t *__restrict__ keys_all,
                                                const uint32_t *__restrict__ vals_all,
                                                uint32_t *__restrict__ keys_out_all,
                                                uint32_t *__restrict__ vals_out_all, int pass,
                                                Control *__restrict__ ctl,
                                                uint32_t *__restrict__ lookback) {
    __shared__ uint32_t s_keys[kSortTile];
    __shared__ uint32_t s_vals[kSortTile];
    __shared__ uint32_t s_whist[W][kDigits];
    __shared__ uint32_t s_tile_start[kDigits];
    __shared__ uint32_t s_out[kDigits];
    __shared__ uint32_t s_warp[W];
    __shared__ uint32_t s_tile;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter[pass], 1u);
    for (int i = tid; i < W * kDigits; i += T) (&s_whist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const TileSpan sp = segs.span(tile);
    const uint32_t n = sp.n, tile_base = sp.base;
    const uint32_t *keys_in = keys_all + sp.start;
    const uint32_t *vals_in = vals_all ? vals_all + sp.start : nullptr;
    uint32_t *keys_out = keys_out_all + sp.start;
    uint32_t *vals_out = vals_out_all + sp.start;
    const int shift = pass * kDigitBits;
    const uint32_t wbase = tile_base + warp * (IPT * 32);

    uint32_t k[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        k[i] = idx < n ? __ldcs(keys_in + idx) : 0u;
    }

    // Global start of this thread's digit: exclusive scan of the pass's digit counts.
    const uint32_t digit_base = block_exclusive_scan(__ldg(sp.hist + tid), s_warp);

    // Stable in-warp ranking, keys visited in input order (item-major, then lane).
    uint32_t rank[IPT / 2];  // two 16-bit ranks per word
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? (k[i] >> shift) & (kDigits - 1) : (uint32_t)kDigits + lane;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        uint32_t cnt = 0;
        if (valid) cnt = s_whist[warp][d];
        __syncwarp();
        if (valid && lane == 31 - __clz(peers)) s_whist[warp][d] = cnt + __popc(peers);
        __syncwarp();
        const uint32_t rk = cnt + __popc(peers & lt);
        if (i & 1) rank[i / 2] |= rk << 16; else rank[i / 2] = rk;
    }
    __syncthreads();

    // Per digit (thread tid): warp-exclusive prefixes and the tile's count.
    uint32_t tile_count = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        const uint32_t c = s_whist[w][tid];
        s_whist[w][tid] = tile_count;
        tile_count += c;
    }

    // Decoupled look-back across tiles for digit tid: read kLookback predecessors at a time
    // (independent loads), then add their counts newest first until a PREFIX is met.
    uint32_t *lb = lookback + (size_t)tile * kDigits + tid;
    uint32_t excl = 0;
    if (tile == sp.first) {
        st_relaxed_gpu(lb, kFlagPrefix | tile_count);
    } else {
        st_relaxed_gpu(lb, kFlagAgg | tile_count);
        long long t0 = 0;
        bool timed = false, done = false;
        int64_t kk = (int64_t)tile - 1;  // next predecessor to add
        while (!done) {
            uint32_t w[kLookback];
#pragma unroll
            for (int i = 0; i < kLookback; ++i)
                w[i] = kk - i >= (int64_t)sp.first ? ld_relaxed_gpu(lookback + (size_t)(kk - i) * kDigits + tid) : kFlagPrefix;
            bool stalled = false;
#pragma unroll
            for (int i = 0; i < kLookback; ++i) {
                if (done || stalled) continue;
                const uint32_t flag = w[i] & ~kCountMask;
                if (flag == 0u) { stalled = true; continue; }
                excl += w[i] & kCountMask;
                --kk;
                if (flag == kFlagPrefix) done = true;
            }
            if (kk < (int64_t)sp.first) done = true;
            if (done || !stalled) continue;
            if (!timed) { t0 = clock64(); timed = true; }
            else if (clock64() - t0 > kSpinLimitCycles ||
                     (ld_relaxed_gpu(&ctl->err) & ERR_LOOKBACK_TIMEOUT)) {
                // give up; once one wait has timed out every other one gives up at once
                atomicOr(&ctl->err, ERR_LOOKBACK_TIMEOUT);
                break;
            }
            __nanosleep(20);
        }
        st_relaxed_gpu(lb, kFlagPrefix | ((excl + tile_count) & kCountMask));
    }

    const uint32_t start = block_exclusive_scan(tile_count, s_warp);
    s_tile_start[tid] = start;
    s_out[tid] = digit_base + excl - start;
    __syncthreads();

    // Stage keys and values in digit order.
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (k[i] >> shift) & (kDigits - 1);
            const uint32_t pos = s_tile_start[d] + s_whist[warp][d] + ((rank[i / 2] >> (16 * (i & 1))) & 0xFFFFu);
            s_keys[pos] = k[i];
            s_vals[pos] = vals_in ? __ldcs(vals_in + idx) : idx;
        }
    }
    __syncthreads();

    const uint32_t tile_n = min((uint32_t)kSortTile, n - tile_base);
    bool oob = false;
    for (uint32_t j = tid; j < tile_n; j += T) {
        const uint32_t key = s_keys[j];
        const uint32_t o = s_out[(key >> shift) & (kDigits - 1)] + j;
        if (o < n) {  // always true unless a look-back wait gave up
            keys_out[o] = key;
            vals_out[o] = s_vals[j];
        } else {
            oob = true;
        }
    }
    if (oob) atomicOr(&ctl->err, ERR_LOOKBACK_TIMEOUT);
}

}  // namespace

void launch_onesweep(const uint32_t *keys_in, const uint32_t *vals_in, uint32_t *keys_out,
                     uint32_t *vals_out, uint32_t n, int pass, Control *ctl, uint32_t *lookback,
                     cudaStream_t s) {
    if (n == 0) return;
    const uint32_t tiles = sort_tiles(n);
    k_onesweep<<<tiles, T, 0, s>>>(OneSegSort{n, &ctl->hist[pass][0]}, keys_in, vals_in, keys_out,
                                   vals_out, pass, ctl, lookback + (size_t)pass * tiles * kDigits);
}

void launch_onesweep_batch(const BatchPlan &bp, const uint32_t *keys_in, const uint32_t *vals_in,
                           uint32_t *keys_out, uint32_t *vals_out, int pass,
                           const uint32_t *seg_hist, Control *ctl, uint32_t *lookback,
                           cudaStream_t s) {
    if (bp.tiles == 0) return;
    k_onesweep<<<bp.tiles, T, 0, s>>>(ManySegSort{bp.rows, bp.tile_seg, seg_hist, pass}, keys_in,
                                      vals_in, keys_out, vals_out, pass, ctl,
                                      lookback + (size_t)pass * bp.tiles * kDigits);
}

}  // namespace lvbh
