// lvbh_device.cuh - device helpers shared by the LBVH build kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace lvbh {

// Bits of the per-build device error word.
enum : uint32_t {
    ERR_NONFINITE = 1u,         // a vertex coordinate is NaN or +-Inf
    ERR_LOOKBACK_TIMEOUT = 2u,  // a decoupled look-back wait exceeded its bound
    ERR_CLIMB = 4u,             // a refit climb exceeded the depth any valid tree has
    ERR_BAD_INDEX = 8u,         // an indexed-mesh vertex index is out of range
    ERR_COPY_TIMEOUT = 16u,     // a copy wait (mbarrier) exceeded its bound
    ERR_SORT_RANGE = 32u,       // a radix sort scatter target fell outside the array (digit
                                // counts inconsistent with the keys, e.g. overlapping calls)
};

// Largest number of cycles a device-side wait spins before it records an error and gives up
// (about a second at B200 clocks); every wait in this library is bounded by it.
constexpr long long kSpinLimitCycles = 2000000000ll;

// split_3 / morton_code of scripts/bvh/kernels/aabb-z-idx.js:197-209: 10 bits per axis
// spread three apart, x in bit 0, y in bit 1, z in bit 2 of each triple.  Inputs above 1023
// keep the bits the masks let through, exactly as the reference's u32 arithmetic does.
__device__ __forceinline__ uint32_t split3(uint32_t x) {
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
__device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
    return split3(x) | (split3(y) << 1) | (split3(z) << 2);
}

// One axis of the quantisation in the reference's operation order (aabb-z-idx.js:191-194):
//   cen = (max + min) * .5f;  rel = (cen - umin) / (umax - umin);  q = u32(rel * 1023.99f)
// Every operation is rounded on its own (no contraction), division is correctly rounded,
// and the float->u32 conversion truncates and saturates (NaN -> 0).
// Split in two for the path that stores centroids before the scene box is known: centroid()
// needs only the triangle, quantise_cen() the scene box; quantise() is the two in a row.
__device__ __forceinline__ float centroid(float bmin, float bmax) { return __fmul_rn(__fadd_rn(bmax, bmin), 0.5f); }
__device__ __forceinline__ uint32_t quantise_cen(float cen, float umin, float umax) {
    const float rel = __fdiv_rn(__fsub_rn(cen, umin), __fsub_rn(umax, umin));
    return __float2uint_rz(__fmul_rn(rel, 1023.99f));
}
__device__ __forceinline__ uint32_t quantise(float bmin, float bmax, float umin, float umax) {
    return quantise_cen(centroid(bmin, bmax), umin, umax);
}

// Common-prefix length delta(i, j) of the sorted keys (radix-tree.js:160-185): -1 when j is
// out of range, clz(k_i ^ k_j) when the keys differ, else 32 + clz(i ^ j) (index tie-break).
// i must be in range.
__device__ __forceinline__ int delta(const uint32_t *__restrict__ keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = __ldg(keys + i), b = __ldg(keys + j);
    return a != b ? __clz(a ^ b) : 32 + __clz(i ^ j);
}

// Monotone float <-> uint32 maps for atomic min/max reductions.  `ord_lo` orders floats
// ascending; atomicMax on ord_hi(x) = ~ord_lo(x) keeps the minimum, atomicMax on ord_lo(x)
// keeps the maximum, so an all-zero word is the identity of both.
__device__ __forceinline__ uint32_t ord_lo(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord_lo_inv(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

__device__ __forceinline__ bool finite3(float4 v) {
    return isfinite(v.x) && isfinite(v.y) && isfinite(v.z);
}

// Acquire-release fences: order this thread's earlier memory operations before its later
// ones for the given scope (the park / merge handshakes need no sequential consistency).
__device__ __forceinline__ void fence_acq_rel_cta() { asm volatile("fence.acq_rel.cta;" ::: "memory"); }
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// Programmatic dependent launch.  A kernel launched by launch_chained starts launching once
// every block of the kernel before it on the stream has exited, before that kernel's
// completion is flushed; chain_wait blocks until the kernel before has completed and its
// memory is visible (and so, transitively, every earlier one).  Every chained kernel calls it
// before its first access to global memory.  Launched the ordinary way it returns at once.
// No kernel signals its dependents early (griddepcontrol.launch_dependents at its start): the
// waiting blocks that let in cost more than the launch they hid (a 2^20-triangle build 0.235
// -> 0.250 ms, against 0.232 ms without the early signal).
__device__ __forceinline__ void chain_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Shared-memory atomic OR with acquire-release semantics at CTA scope: the caller's earlier
// writes are visible to a thread that later sees its bit, and what the caller reads after it
// includes the writes of threads whose bits it saw.
__device__ __forceinline__ uint32_t atom_or_acq_rel_cta(uint32_t *p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.cta.shared.or.b32 %0, [%1], %2;"
                 : "=r"(old) : "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(v) : "memory");
    return old;
}

// Global-memory atomic exchange with acquire-release semantics at GPU scope (the park / merge
// handshake across CTAs, as atom_or_acq_rel_cta is within one).
__device__ __forceinline__ uint32_t atom_exch_acq_rel_gpu(uint32_t *p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.exch.b32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Relaxed gpu-scope load / store of a 32-bit word another CTA publishes.
__device__ __forceinline__ uint32_t ld_relaxed_gpu(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_gpu(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// 16-byte asynchronous copy global -> shared (L2 only), its group commit and wait.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
// 4-byte asynchronous copy global -> shared (cached at all levels): a scattered destination per
// thread, no register held while it is in flight.
__device__ __forceinline__ void cp_async4(void *smem_dst, const void *gmem_src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// TMA copies global -> shared completing on an mbarrier in this CTA's shared memory.  A random
// gather of rows from DRAM runs far faster this way than through per-thread 16-byte cp.async:
// on the B200 a gather of 16.7 M random 48-byte rows into shared memory took 1.14 ms as three
// cp.async per row, 0.67 ms as one 48-byte bulk copy per row and 0.55 ms as one tile::gather4
// copy per four rows through a tensor map with 64-byte L2 fills.  For 16-byte rows that hit L2
// cp.async stays ahead (less work per copy).  No multicast.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// makes initialised mbarriers visible to the copy engine; a CTA barrier follows before use
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// one arrival that also raises the phase's expected byte count
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// Four rows of a 2-D tensor (rows r0..r3, the tensor map's one-row box from column 0) into
// consecutive shared memory by one TMA tile::gather4 copy, completing on an mbarrier.  The
// destination starts on a 128-byte boundary; the rows are inside the tensor.  No multicast.
__device__ __forceinline__ void gather4_g2s(void *smem_dst, const void *tensor_map, uint32_t r0, uint32_t r1,
                                            uint32_t r2, uint32_t r3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        ::"r"(smem_addr(smem_dst)), "l"(reinterpret_cast<uint64_t>(tensor_map)), "r"(0), "r"(r0), "r"(r1), "r"(r2),
          "r"(r3), "r"(smem_addr(bar))
        : "memory");
}
// Waits for the completion of the mbarrier phase of the given parity, at most kSpinLimitCycles;
// false if the bound ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    long long t0 = 0;
    for (uint32_t it = 0;; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
        if (ok) return true;
        if (it == 0) t0 = clock64();
        else if (clock64() - t0 > kSpinLimitCycles) return false;
    }
}

// Streaming (evict-first) 16-byte load and store.
__device__ __forceinline__ float4 ld_stream(const float4 *p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(float4 *p, float4 v) { __stcs(p, v); }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Adds one count per valid lane to the shared-memory histogram h at bin d, one atomic per run
// of equal bins over consecutive lanes: the run's first lane adds its length.  Input in
// spatially coherent order (a mesh's triangles, keys grouped by the previous sort digit) gives
// long runs, which plain per-lane atomics would serialise on one bin.  All 32 lanes call it.
// True when the warp's bins d form at most 8 runs over consecutive lanes (warp-uniform): the
// case add_runs pays for; scattered bins are cheaper with one atomic per lane.
__device__ __forceinline__ bool runs_few(uint32_t d, bool valid) {
    const int lane = threadIdx.x & 31;
    const uint32_t dv = valid ? d : 0xFFFFFFFFu;
    const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, dv, 1);
    return __popc(__ballot_sync(0xFFFFFFFFu, lane == 0 || dv != up)) <= 8;
}

__device__ __forceinline__ void add_runs(uint32_t *h, uint32_t d, bool valid) {
    const int lane = threadIdx.x & 31;
    const uint32_t dv = valid ? d : 0xFFFFFFFFu;  // invalid lanes form runs of their own
    const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, dv, 1);
    const bool head = lane == 0 || dv != up;
    const uint32_t heads = __ballot_sync(0xFFFFFFFFu, head);
    if (head && valid) {
        const uint32_t after = heads & ~((2u << lane) - 1u);  // heads of the lanes above
        const int next = after ? __ffs(after) - 1 : 32;
        atomicAdd(h + d, (uint32_t)(next - lane));
    }
}

}  // namespace lvbh
