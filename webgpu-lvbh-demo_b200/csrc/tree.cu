// tree.cu - K3: Karras radix tree over the sorted Morton keys -> parent links (sm_100a).
//
// Restates compute_radix_tree_pointers / compute_child_index (scripts/bvh/kernels/
// radix-tree.js:137-238): one thread per internal node i in [0, N-2] finds the direction
// d = sign(delta(i, i+1) - delta(i, i-1)), bounds and binary-searches its range end j, then
// binary-searches the split gamma; children gamma / gamma+1 are leaves when they are the range
// ends.  The reference's split loop keeps testing t = 1 after the search has converged until
// its i32 step overflows; those extra tests can never move s (s is already the largest
// offset whose prefix exceeds delta_node), so the loop here stops at the first t == 1.
// delta is __clz of the key XOR, with the index tie-break for equal keys.
//
// Output layout (radix-tree.js:57-60,146-156): parents[child] = i for internal children,
// parents[N + leaf] = i for leaves; slots 0 (root) and N-1 (unused) are written as 0.
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

__global__ void __launch_bounds__(256) k_tree(const uint32_t *__restrict__ keys, int n,
                                              int32_t *__restrict__ parents,
                                              uint32_t *__restrict__ epoch) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i == 0) {
        parents[0] = 0;
        parents[n - 1] = 0;
        // New arrival epoch for K4 (see refit.cu); 0 is the value a fresh flag array holds.
        const uint32_t e = *epoch + 1u;
        *epoch = e == 0u ? 1u : e;
    }
    if (i >= n - 1) return;

    const int d = delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1) > 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t > 0; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int s = 0;
    for (int div = 2;; div <<= 1) {
        const int t = (l + div - 1) / div;  // ceil(l / div), as (l - 1 + v) / v in the reference
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    parents[lo == gamma ? n + gamma : gamma] = i;
    parents[hi == gamma + 1 ? n + gamma + 1 : gamma + 1] = i;
}

}  // namespace

void launch_tree(const uint32_t *keys, uint32_t n, int32_t *parents, uint32_t *epoch,
                 cudaStream_t s) {
    if (n < 2) return;
    k_tree<<<(n - 1 + 255) / 256, 256, 0, s>>>(keys, (int)n, parents, epoch);
}

}  // namespace lvbh
