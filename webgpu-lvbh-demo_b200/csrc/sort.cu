// sort.cu - K2: onesweep stable LSD radix sort pass of (Morton key, triangle index) (sm_100a).
//
// Replaces the reference's 2-bit x 16-pass sort (scripts/bvh/kernels/radix-sort.js:162-499:
// init_idx, init_off, two scan_up levels and scan_and_sort per pass, 64 submits and 16 host
// waits).  Its result is the stable argsort of the keys - ties keep ascending input index -
// and this pass keeps that contract.  The build's keys have 30 bits, sorted in three passes of
// 10-bit digits; full 32-bit keys (the allocation-free entry point) take four 8-bit passes.
//
//   * the global digit counts of a pass are summed by its tile-histogram kernel (pass 0's by the
//     Morton kernel, which writes pass 0's tile histograms with the keys);
//   * a tile of 4096 keys (256 threads x 16) is ranked in shared memory: each warp walks its
//     keys in input order; the lanes holding the same digit (its peers) are found with one
//     ballot per digit bit, and the peers' lane order plus a per-warp running count in a
//     16-bit shared counter gives each key its stable rank;
//   * the tile's digit counts are combined with earlier tiles by decoupled look-back: tiles
//     are numbered by an atomic counter in launch order, each publishes its counts (flag
//     AGGREGATE) and then its inclusive prefix (flag PREFIX) in one 32-bit word per digit, and
//     looks back only at tiles that have already started, so the waits always end;
//   * every wait is bounded (kSpinLimitCycles, or the control block's test bound); past it the
//     kernel records ERR_LOOKBACK_TIMEOUT and carries on, so it never hangs, and the tree
//     kernels that follow in a build see the flag and build nothing from the unfinished sort;
//   * keys and values are staged in digit order in shared memory and written out so that
//     consecutive threads write consecutive addresses of each digit's run.
//
// The plain build sorts one array of up to 2^29 keys, thousands of tiles long.  There a
// look-back over 1024 digits would read 4 KB per predecessor tile and walk back about half a
// wave of resident tiles, so its pass runs reduce-then-scan instead, with no waits at all:
//   k_tile_hist   per tile of 4096 keys its digit counts, per chunk of 8 tiles their sum;
//   k_chunk_scan  per chunk and digit the global output offset of the chunk's first key
//                 (exclusive scan over chunks plus the digit's global start);
//   k_scatter     ranks its tile as above, adds the counts of the earlier tiles of its chunk
//                 (at most 7 rows of 4 KB, already final) to the chunk offset, and scatters.
// The batched build's segments span at most 64 tiles, so it keeps the one-kernel look-back.
//
// HBM-bound: per key one 4-byte key read (+4-byte value read after the first pass) and two
// 4-byte writes (+ the 4-byte key read of k_tile_hist when reducing first).
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
constexpr int kLookback = 4;  // predecessor tiles read per look-back step and digit

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

template <int BITS>
struct ManySegSort {
    const SegRow *rows;
    const uint32_t *tile_seg;
    const uint32_t *seg_hist;  // kHistWords per segment: [pass][digit]
    int pass;
    __device__ __forceinline__ TileSpan span(uint32_t tile) const {
        const uint32_t sg = __ldg(tile_seg + tile);
        const uint32_t t0 = __ldg(&rows[sg].tri), t1 = __ldg(&rows[sg + 1].tri);
        const uint32_t first = __ldg(&rows[sg].tile);
        return TileSpan{t0, t1 - t0, (tile - first) * (uint32_t)kSortTile, first,
                        seg_hist + (size_t)sg * kHistWords + pass * (1 << BITS)};
    }
};

template <int BITS>
struct SortSmem {
    static constexpr int D = 1 << BITS;
    uint32_t keys[kSortTile];
    uint32_t vals[kSortTile];
    uint16_t whist[W][D];  // per-warp digit counts, then per-warp staging offsets
    uint32_t out[D];       // output position of staged index 0 of each digit
    uint32_t warp[W];
    uint32_t tile;
};

template <int BITS, class Segs>
__global__ void __launch_bounds__(T, 4) k_onesweep(Segs segs, const uint32_t *__restrict__ keys_all,
                                                const uint32_t *__restrict__ vals_all,
                                                uint32_t *__restrict__ keys_out_all,
                                                uint32_t *__restrict__ vals_out_all, int pass,
                                                Control *__restrict__ ctl,
                                                uint32_t *__restrict__ lookback) {
    constexpr int D = 1 << BITS;
    constexpr int P = D / T;  // digits per thread in the per-digit phases (contiguous)
    static_assert(P >= 1 && P * T == D, "digits per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<BITS> &S = *reinterpret_cast<SortSmem<BITS> *>(smem_raw);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) S.tile = atomicAdd(&ctl->tile_counter[pass], 1u);
    // test hook words (zero in normal use): a tile that publishes nothing, the wait bound
    const uint32_t stall1 = ctl->test_stall_tile1;
    const long long spin_limit = ctl->test_spin_limit ? (long long)ctl->test_spin_limit : kSpinLimitCycles;
    for (int i = tid; i < W * D / 2; i += T) reinterpret_cast<uint32_t *>(&S.whist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = S.tile;
    const TileSpan sp = segs.span(tile);
    const uint32_t n = sp.n, tile_base = sp.base;
    const uint32_t *keys_in = keys_all + sp.start;
    const uint32_t *vals_in = vals_all ? vals_all + sp.start : nullptr;
    uint32_t *keys_out = keys_out_all + sp.start;
    uint32_t *vals_out = vals_out_all + sp.start;
    const int shift = pass * BITS;
    const uint32_t wbase = tile_base + warp * (IPT * 32);

    uint32_t k[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        k[i] = idx < n ? __ldcs(keys_in + idx) : 0u;
    }
    // the values are read only when they are staged: start bringing them into L2 now
    if (vals_in && lane < IPT && wbase + lane * 32 < n)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(vals_in + wbase + lane * 32));

    // Stable in-warp ranking, keys visited in input order (item-major, then lane).
    uint32_t rank[IPT / 2];  // two 16-bit ranks per word
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = (k[i] >> shift) & (D - 1);
        uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
        for (int b = 0; b < BITS; ++b) {
            const uint32_t bit = (d >> b) & 1u;
            const uint32_t vote = __ballot_sync(0xFFFFFFFFu, bit);
            peers &= bit ? vote : ~vote;
        }
        uint32_t cnt = 0;
        if (valid) cnt = S.whist[warp][d];
        __syncwarp();
        if (valid && lane == 31 - __clz(peers)) S.whist[warp][d] = (uint16_t)(cnt + __popc(peers));
        __syncwarp();
        const uint32_t rk = cnt + __popc(peers & lt);
        if (i & 1) rank[i / 2] |= rk << 16; else rank[i / 2] = rk;
    }
    __syncthreads();

    // Per digit (thread tid owns digits tid*P .. tid*P+P-1): warp-exclusive prefixes (in place)
    // and the tile's counts.
    uint32_t cnt[P];
#pragma unroll
    for (int j = 0; j < P; ++j) {
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const uint32_t x = S.whist[w][tid * P + j];
            S.whist[w][tid * P + j] = (uint16_t)c;
            c += x;
        }
        cnt[j] = c;
    }

    // Publish the tile's counts at once (its inclusive prefix when it is the segment's first
    // tile), so that later tiles can look back past it while it stages its keys.
    uint32_t *lb = lookback + (size_t)tile * D + tid * P;
    const bool first = tile == sp.first;
    const bool publish = tile + 1u != stall1;
#pragma unroll
    for (int j = 0; j < P; ++j)
        if (publish) st_relaxed_gpu(lb + j, (first ? kFlagPrefix : kFlagAgg) | cnt[j]);

    // The tile's start of each digit in the staging buffer (exclusive scan of its counts).
    uint32_t tst[P], tsum = 0;
#pragma unroll
    for (int j = 0; j < P; ++j) tsum += cnt[j];
    uint32_t tstart = block_exclusive_scan(tsum, S.warp);
#pragma unroll
    for (int j = 0; j < P; ++j) {
        const int dg = tid * P + j;
        tst[j] = tstart;
#pragma unroll
        for (int w = 0; w < W; ++w) S.whist[w][dg] = (uint16_t)(S.whist[w][dg] + tstart);
        tstart += cnt[j];
    }
    __syncthreads();

    // Stage keys and values in digit order (values by 4-byte asynchronous copies, in flight
    // during the look-back).
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (k[i] >> shift) & (D - 1);
            const uint32_t pos = S.whist[warp][d] + ((rank[i / 2] >> (16 * (i & 1))) & 0xFFFFu);
            S.keys[pos] = k[i];
            if (vals_in) cp_async4(&S.vals[pos], vals_in + idx);
            else S.vals[pos] = idx;
        }
    }
    cp_async_commit();

    // Decoupled look-back across tiles, all P digits together: read kLookback predecessors
    // per digit at a time (independent loads), add their counts newest first until a PREFIX.
    uint32_t excl[P];
#pragma unroll
    for (int j = 0; j < P; ++j) excl[j] = 0;
    if (!first) {
        int kk[P];
#pragma unroll
        for (int j = 0; j < P; ++j) kk[j] = (int)tile - 1;  // next predecessor to add
        uint32_t done = 0;
        constexpr uint32_t kAll = (1u << P) - 1u;
        long long t0 = 0;
        bool timed = false;
        while (done != kAll) {
            uint32_t w[P][kLookback];
#pragma unroll
            for (int j = 0; j < P; ++j)
#pragma unroll
                for (int i = 0; i < kLookback; ++i)
                    w[j][i] = (!(done >> j & 1u) && kk[j] - i >= (int)sp.first)
                                  ? ld_relaxed_gpu(lookback + (size_t)(kk[j] - i) * D + tid * P + j)
                                  : kFlagPrefix;
            bool stalled = false;
#pragma unroll
            for (int j = 0; j < P; ++j) {
                bool stop = (done >> j & 1u) != 0;
#pragma unroll
                for (int i = 0; i < kLookback; ++i) {
                    if (stop) continue;
                    const uint32_t flag = w[j][i] & ~kCountMask;
                    if (flag == 0u) { stop = true; stalled = true; continue; }
                    excl[j] += w[j][i] & kCountMask;
                    --kk[j];
                    if (flag == kFlagPrefix) { stop = true; done |= 1u << j; }
                }
                if (kk[j] < (int)sp.first) done |= 1u << j;
            }
            if (done == kAll || !stalled) continue;
            if (!timed) { t0 = clock64(); timed = true; }
            else if (clock64() - t0 > spin_limit ||
                     (ld_relaxed_gpu(&ctl->err) & ERR_LOOKBACK_TIMEOUT)) {
                // give up; once one wait has timed out every other one gives up at once
                atomicOr(&ctl->err, ERR_LOOKBACK_TIMEOUT);
                break;
            }
            __nanosleep(20);
        }
#pragma unroll
        for (int j = 0; j < P; ++j)
            if (publish) st_relaxed_gpu(lb + j, kFlagPrefix | ((excl[j] + cnt[j]) & kCountMask));
    }

    // Global start of each digit: exclusive scan of the pass's counts.
    uint32_t g[P], gsum = 0;
#pragma unroll
    for (int j = 0; j < P; ++j) { g[j] = __ldg(sp.hist + tid * P + j); gsum += g[j]; }
    uint32_t gbase = block_exclusive_scan(gsum, S.warp);
#pragma unroll
    for (int j = 0; j < P; ++j) {
        S.out[tid * P + j] = gbase + excl[j] - tst[j];
        gbase += g[j];
    }
    cp_async_wait_all();
    __syncthreads();

    const uint32_t tile_n = min((uint32_t)kSortTile, n - tile_base);
    bool oob = false;
    for (uint32_t j = tid; j < tile_n; j += T) {
        const uint32_t key = S.keys[j];
        const uint32_t o = S.out[(key >> shift) & (D - 1)] + j;
        if (o < n) {  // always true unless a look-back wait gave up or the counts are wrong
            keys_out[o] = key;
            vals_out[o] = S.vals[j];
        } else {
            oob = true;
        }
    }
    if (oob) atomicOr(&ctl->err, ERR_SORT_RANGE);
}


// Reduce: digit counts of every tile (tile_hist[tile][digit]) and of every chunk of chunk_tiles
// tiles (chunk_sum[chunk][digit]), added up into the pass's global counts (ghist: kHistParts
// partial rows, zero before; the chunk goes to row chunk % kHistParts).  One block per chunk;
// each thread owns P contiguous digits.
template <int BITS>
__global__ void __launch_bounds__(T) k_tile_hist(const uint32_t *__restrict__ keys, uint32_t n, int pass,
                                                 uint32_t chunk_tiles, uint32_t *__restrict__ tile_hist,
                                                 uint32_t *__restrict__ chunk_sum, uint32_t *__restrict__ ghist) {
    constexpr int D = 1 << BITS, P = D / T;
    __shared__ __align__(16) uint32_t h[D];
    const int tid = threadIdx.x, shift = pass * BITS;
    chain_wait();
    const uint32_t tiles = sort_tiles(n);
    uint32_t acc[P];
#pragma unroll
    for (int j = 0; j < P; ++j) acc[j] = 0;
    // the next tile's keys are loaded while this one is counted
    uint32_t kn[IPT];
    auto load = [&](uint32_t tile) {
        const uint32_t base = tile * (uint32_t)kSortTile;
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const uint32_t idx = base + i * T + tid;
            kn[i] = idx < n ? __ldcs(keys + idx) : 0xFFFFFFFFu;
        }
    };
    if (blockIdx.x * chunk_tiles < tiles) load(blockIdx.x * chunk_tiles);
    for (uint32_t tt = 0; tt < chunk_tiles; ++tt) {
        const uint32_t tile = blockIdx.x * chunk_tiles + tt;
        if (tile >= tiles) break;  // uniform across the block
        uint32_t k[IPT];
#pragma unroll
        for (int i = 0; i < IPT; ++i) k[i] = kn[i];
        if (tt + 1 < chunk_tiles && tile + 1 < tiles) load(tile + 1);
        for (int i = tid; i < D; i += T) h[i] = 0;
        __syncthreads();
        const uint32_t base = tile * (uint32_t)kSortTile;
        // keys grouped by the previous digit repeat this one over long runs when the input was
        // spatially coherent; the warp tests its first 32 keys and keeps the answer for the tile
        const bool coherent = runs_few((k[0] >> shift) & (D - 1), base + tid < n);
#pragma unroll
        for (int i = 0; i < IPT; ++i) {
            const uint32_t d = (k[i] >> shift) & (D - 1);
            const bool valid = base + i * T + tid < n;
            if (coherent) add_runs(h, d, valid);
            else if (valid) atomicAdd(&h[d], 1u);
        }
        __syncthreads();
        uint32_t c[P];
#pragma unroll
        for (int j = 0; j < P; ++j) { c[j] = h[tid * P + j]; acc[j] += c[j]; }
        uint32_t *row = tile_hist + (size_t)tile * D + tid * P;
#pragma unroll
        for (int j = 0; j < P; ++j) row[j] = c[j];
        __syncthreads();
    }
    uint32_t *row = chunk_sum + (size_t)blockIdx.x * D + tid * P;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        row[j] = acc[j];
        if (acc[j]) atomicAdd(ghist + (blockIdx.x % kHistParts) * D + tid * P + j, acc[j]);
    }
}

// Scan: chunk_off[c][d] = start of digit d in the pass's output (exclusive scan of the global
// counts over digits, the kHistParts partial rows of ghist summed) + counts of digit d in chunks
// before c.  Block b covers digits
// 32b .. 32b+31 (lane = digit); its 32 warps split the chunks.
constexpr int kScanThreads = 1024;
template <int BITS>
__global__ void __launch_bounds__(kScanThreads) k_chunk_scan(const uint32_t *__restrict__ chunk_sum,
                                                             uint32_t chunks,
                                                             const uint32_t *__restrict__ ghist,
                                                             uint32_t *__restrict__ chunk_off) {
    constexpr int D = 1 << BITS, SW = kScanThreads / 32;
    static_assert(D == kScanThreads, "one digit per thread in the digit scan");
    __shared__ uint32_t s_wsum[SW];
    __shared__ uint32_t s_base[32];
    __shared__ uint32_t s_part[SW][32];
    chain_wait();
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // digit starts: exclusive scan of the global counts, one digit per thread
    uint32_t g = 0;
#pragma unroll
    for (int r = 0; r < kHistParts; ++r) g += __ldg(ghist + r * D + tid);
    uint32_t incl = g;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    uint32_t woff = 0;
    for (int w = 0; w < warp; ++w) woff += s_wsum[w];
    const int d0 = blockIdx.x * 32;
    if (tid >= d0 && tid < d0 + 32) s_base[tid - d0] = woff + incl - g;
    const uint32_t per = (chunks + SW - 1) / SW;
    const uint32_t c0 = warp * per, c1 = min(chunks, c0 + per);
    const int d = d0 + lane;
    uint32_t sum = 0;
    for (uint32_t c = c0; c < c1; ++c) sum += __ldg(chunk_sum + (size_t)c * D + d);
    s_part[warp][lane] = sum;
    __syncthreads();
    uint32_t off = s_base[lane];
    for (int w = 0; w < warp; ++w) off += s_part[w][lane];
    for (uint32_t c = c0; c < c1; ++c) {
        chunk_off[(size_t)c * D + d] = off;
        off += __ldg(chunk_sum + (size_t)c * D + d);
    }
}

// Scatter: the ranking and staging of k_onesweep; the prefix of each digit is the chunk's
// offset plus the counts of the chunk's earlier tiles.  Tile = blockIdx.x, no waits.
template <int BITS>
__global__ void __launch_bounds__(T, 4) k_scatter(const uint32_t *__restrict__ keys_in,
                                               const uint32_t *__restrict__ vals_in,
                                               uint32_t *__restrict__ keys_out,
                                               uint32_t *__restrict__ vals_out, uint32_t n,
                                               int pass, const uint32_t *__restrict__ tile_hist,
                                               const uint32_t *__restrict__ chunk_off,
                                               uint32_t chunk_tiles, Control *__restrict__ ctl) {
    constexpr int D = 1 << BITS;
    constexpr int P = D / T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<BITS> &S = *reinterpret_cast<SortSmem<BITS> *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // each warp clears its own counts: the ranking below touches only those, so the warp starts it
    // without waiting for the block (a block barrier there cost about 1 us of the three passes)
    for (int i = lane; i < D / 2; i += 32) reinterpret_cast<uint32_t *>(&S.whist[warp][0])[i] = 0;
    chain_wait();
    const uint32_t tile = blockIdx.x, tile_base = tile * (uint32_t)kSortTile;
    const int shift = pass * BITS;
    const uint32_t wbase = tile_base + warp * (IPT * 32);

    uint32_t k[IPT];
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        k[i] = idx < n ? __ldcs(keys_in + idx) : 0u;
    }
    // the tile's values are read only when they are staged, after the ranking: start bringing
    // them into L2 now (one 128-byte line of 32 values per lane)
    if (vals_in && lane < IPT && wbase + lane * 32 < n)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(vals_in + wbase + lane * 32));
    // the digit prefixes of this tile (final values: independent 16-byte loads, all in flight
    // with the keys), parked in S.out until the tile's own starts are known
    {
        static_assert(P == 4, "one 16-byte load per row");
        const uint32_t chunk = tile / chunk_tiles, t0c = chunk * chunk_tiles;
        uint4 acc = __ldg(reinterpret_cast<const uint4 *>(chunk_off + (size_t)chunk * D + tid * P));
        uint4 row[kSortChunkTiles - 1];
#pragma unroll
        for (int q = 0; q < kSortChunkTiles - 1; ++q)
            row[q] = t0c + q < tile ? __ldg(reinterpret_cast<const uint4 *>(tile_hist + (size_t)(t0c + q) * D + tid * P))
                                    : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
        for (int q = 0; q < kSortChunkTiles - 1; ++q) {
            acc.x += row[q].x; acc.y += row[q].y; acc.z += row[q].z; acc.w += row[q].w;
        }
        const uint32_t pre[P] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
        for (int j = 0; j < P; ++j) S.out[tid * P + j] = pre[j];  // read after the barriers below
    }
    __syncwarp();

    uint32_t rank[IPT / 2];
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = (k[i] >> shift) & (D - 1);
        uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
        for (int b = 0; b < BITS; ++b) {
            const uint32_t bit = (d >> b) & 1u;
            const uint32_t vote = __ballot_sync(0xFFFFFFFFu, bit);
            peers &= bit ? vote : ~vote;
        }
        uint32_t cnt = 0;
        if (valid) cnt = S.whist[warp][d];
        __syncwarp();
        if (valid && lane == 31 - __clz(peers)) S.whist[warp][d] = (uint16_t)(cnt + __popc(peers));
        __syncwarp();
        const uint32_t rk = cnt + __popc(peers & lt);
        if (i & 1) rank[i / 2] |= rk << 16; else rank[i / 2] = rk;
    }
    __syncthreads();

    uint32_t cnt[P], tsum = 0;
#pragma unroll
    for (int j = 0; j < P; ++j) {
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            const uint32_t x = S.whist[w][tid * P + j];
            S.whist[w][tid * P + j] = (uint16_t)c;
            c += x;
        }
        cnt[j] = c;
        tsum += c;
    }
    uint32_t tstart = block_exclusive_scan(tsum, S.warp);
#pragma unroll
    for (int j = 0; j < P; ++j) {
        const int dg = tid * P + j;
#pragma unroll
        for (int w = 0; w < W; ++w) S.whist[w][dg] = (uint16_t)(S.whist[w][dg] + tstart);
        S.out[dg] -= tstart;
        tstart += cnt[j];
    }
    __syncthreads();

    // the values go straight from global memory to their staged slots by 4-byte asynchronous
    // copies: all of a thread's copies are in flight at once and hold no registers (loads
    // followed by shared stores waited for each value in turn)
#pragma unroll
    for (int i = 0; i < IPT; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (k[i] >> shift) & (D - 1);
            const uint32_t pos = S.whist[warp][d] + ((rank[i / 2] >> (16 * (i & 1))) & 0xFFFFu);
            S.keys[pos] = k[i];
            if (vals_in) cp_async4(&S.vals[pos], vals_in + idx);
            else S.vals[pos] = idx;
        }
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();

    const uint32_t tile_n = min((uint32_t)kSortTile, n - tile_base);
    bool oob = false;
    for (uint32_t j = tid; j < tile_n; j += T) {
        const uint32_t key = S.keys[j];
        const uint32_t o = S.out[(key >> shift) & (D - 1)] + j;
        if (o < n) {  // always true for consistent counts
            keys_out[o] = key;
            vals_out[o] = S.vals[j];
        } else {
            oob = true;
        }
    }
    if (oob) atomicOr(&ctl->err, ERR_SORT_RANGE);
}

template <int BITS, class Segs>
void launch(Segs segs, uint32_t tiles, const uint32_t *keys_in, const uint32_t *vals_in,
            uint32_t *keys_out, uint32_t *vals_out, int pass, Control *ctl, uint32_t *lookback,
            cudaStream_t s) {
    k_onesweep<BITS, Segs><<<tiles, T, sizeof(SortSmem<BITS>), s>>>(
        segs, keys_in, vals_in, keys_out, vals_out, pass, ctl, lookback);
}

template <int BITS, class Segs>
cudaError_t allow_smem() {
    return cudaFuncSetAttribute(k_onesweep<BITS, Segs>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(SortSmem<BITS>));
}

}  // namespace

cudaError_t sort_init() {
    cudaError_t e = allow_smem<kDigitBits, ManySegSort<kDigitBits>>();
    if (e == cudaSuccess) e = allow_smem<kDigitBits32, ManySegSort<kDigitBits32>>();
    if (e == cudaSuccess) e = allow_smem<kDigitBits32, OneSegSort>();
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_scatter<kDigitBits>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(SortSmem<kDigitBits>));
    return e;
}

size_t sort_scratch_words(uint32_t n) { return ((size_t)sort_tiles(n) + 2ull * sort_chunks_bound(n)) * kDigits; }

void launch_sort_pass(const uint32_t *keys_in, const uint32_t *vals_in, uint32_t *keys_out,
                      uint32_t *vals_out, uint32_t n, int pass, bool counted, Control *ctl,
                      uint32_t *scratch, cudaStream_t s) {
    if (n == 0) return;
    const uint32_t tiles = sort_tiles(n), chunks = sort_chunks(n);
    uint32_t *tile_hist = scratch;
    uint32_t *chunk_sum = sort_chunk_sums(scratch, n);
    uint32_t *chunk_off = chunk_sum + (size_t)chunks * kDigits;
    const uint32_t ct = sort_chunk_tiles(n);
    uint32_t *ghist = &ctl->hist_part[pass][0][0];
    const bool chain = chain_build(n);
    if (!counted)
        launch_chained(chain, k_tile_hist<kDigitBits>, chunks, T, 0, s, keys_in, n, pass, ct, tile_hist, chunk_sum, ghist);
    launch_chained(chain, k_chunk_scan<kDigitBits>, kDigits / 32, kScanThreads, 0, s, chunk_sum, chunks, ghist, chunk_off);
    launch_chained(chain, k_scatter<kDigitBits>, tiles, T, sizeof(SortSmem<kDigitBits>), s, keys_in, vals_in, keys_out,
                   vals_out, n, pass, tile_hist, chunk_off, ct, ctl);
}

void launch_onesweep32(const uint32_t *keys_in, const uint32_t *vals_in, uint32_t *keys_out,
                       uint32_t *vals_out, uint32_t n, int pass, Control *ctl, uint32_t *lookback,
                       cudaStream_t s) {
    if (n == 0) return;
    const uint32_t tiles = sort_tiles(n);
    launch<kDigitBits32>(OneSegSort{n, ctl->hist + pass * kDigits32}, tiles, keys_in, vals_in,
                         keys_out, vals_out, pass, ctl, lookback + (size_t)pass * tiles * kDigits32, s);
}

void launch_onesweep_batch(const BatchPlan &bp, const uint32_t *keys_in, const uint32_t *vals_in,
                           uint32_t *keys_out, uint32_t *vals_out, int pass,
                           const uint32_t *seg_hist, Control *ctl, uint32_t *lookback,
                           cudaStream_t s) {
    if (bp.tiles == 0) return;
    if (bp.digit_bits == kDigitBits32)
        launch<kDigitBits32>(ManySegSort<kDigitBits32>{bp.rows, bp.tile_seg, seg_hist, pass}, bp.tiles,
                             keys_in, vals_in, keys_out, vals_out, pass, ctl,
                             lookback + (size_t)pass * bp.tiles * kDigits32, s);
    else
        launch<kDigitBits>(ManySegSort<kDigitBits>{bp.rows, bp.tile_seg, seg_hist, pass}, bp.tiles,
                           keys_in, vals_in, keys_out, vals_out, pass, ctl,
                           lookback + (size_t)pass * bp.tiles * kDigits, s);
}

}  // namespace lvbh
