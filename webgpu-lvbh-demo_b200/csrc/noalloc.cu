// noalloc.cu - lvbh_sort_pairs_noalloc: the build's stable radix sort of (key, index) for
// callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc at the point where they need a sort: a
// render or serving loop that must not stall between frames (cudaMalloc / cudaFree
// synchronise the device), a process that has already handed its whole memory budget to its
// own pool, or a plugin host that owns every device allocation.  They pass the input keys and
// the two output arrays; everything else the sort needs - the ping-pong keys and values, the
// digit histograms, the decoupled look-back words and the error word - lives in one
// file-scope device array, g_scratch, sized for kMaxKeys keys.  Every GPU that loads the
// library holds that array (about 9.6 MB) until the process exits.
//
// In host code the name g_scratch is a host-side stand-in, not a device address: handing it
// to a kernel would fault, or silently use the wrong memory where the GPU can reach host
// memory.  The first call on each device therefore resolves the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that first call before
// any stream capture.  Each call clears the parts that must start at zero (histograms, tile
// counters, look-back words, error word) with cudaMemsetAsync on the caller's stream.  All
// calls on a device share the one array: calls that overlap on the GPU (different streams
// without ordering between them, or different host threads) race and corrupt each other.
// No cudaMalloc, cudaFree or allocating library routine is called.
#include <cstddef>
#include <cstring>
#include <mutex>

#include "lvbh.h"
#include "lvbh_device.cuh"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

constexpr uint32_t kMaxKeys = LVBH_NOALLOC_MAX_KEYS;
constexpr uint32_t kMaxTiles = (kMaxKeys + kSortTile - 1) / kSortTile;
constexpr size_t kControlWords = (sizeof(Control) + 255) / 256 * 256 / 4;
constexpr size_t kLookbackWords = (size_t)kSortPasses32 * kMaxTiles * kDigits32;
constexpr size_t kScratchWords = kControlWords + kLookbackWords + 2ull * kMaxKeys;

// Scratch of the allocation-free sort: [Control][look-back words][keys][values].
static __device__ __align__(256) uint32_t g_scratch[kScratchWords];

// Digit histograms of all four 8-bit passes of full 32-bit keys.
__global__ void __launch_bounds__(256) k_digit_hist(const uint32_t *__restrict__ keys, uint32_t n,
                                                    Control *__restrict__ ctl) {
    __shared__ uint32_t hist[kSortPasses32][kDigits32];
    for (int i = threadIdx.x; i < kSortPasses32 * kDigits32; i += 256) (&hist[0][0])[i] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const uint32_t key = __ldg(keys + i);
#pragma unroll
        for (int p = 0; p < kSortPasses32; ++p)
            atomicAdd(&hist[p][(key >> (kDigitBits32 * p)) & (kDigits32 - 1)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kSortPasses32 * kDigits32; i += 256) {
        const uint32_t c = (&hist[0][0])[i];
        if (c) atomicAdd(ctl->hist + i, c);
    }
}

std::mutex g_mutex;
void *g_addr[64] = {};  // device address of g_scratch, per device ordinal

}  // namespace

}  // namespace lvbh

using namespace lvbh;

extern "C" int lvbh_sort_pairs_noalloc(const uint32_t *keys_in, uint32_t num_keys,
                                       uint32_t *keys_out, uint32_t *perm_out, void *stream) {
    if (num_keys > kMaxKeys) return LVBH_ERANGE;
    if (num_keys == 0) return LVBH_OK;
    if (!keys_in || !keys_out || !perm_out) return LVBH_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return LVBH_ECUDA;
    }
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_addr[dev]) {  // set-up, once per device, with that device current
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return LVBH_ECUDA;
            }
            if (sort_init() != cudaSuccess) {
                cudaGetLastError();
                return LVBH_ECUDA;
            }
            g_addr[dev] = p;
        }
        base = g_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t *words = static_cast<uint32_t *>(base);
    Control *ctl = reinterpret_cast<Control *>(words);
    uint32_t *lookback = words + kControlWords;
    uint32_t *keys_b = lookback + kLookbackWords;
    uint32_t *vals_b = keys_b + kMaxKeys;
    // what must start at zero: the error words, tile counters, histograms and look-back words
    const size_t zero_bytes = (kControlWords + (size_t)kSortPasses32 * sort_tiles(num_keys) * kDigits32) * 4;
    if (cudaMemsetAsync(words, 0, zero_bytes, s) != cudaSuccess) { cudaGetLastError(); return LVBH_ECUDA; }
    int blocks = (int)((num_keys + 255) / 256);
    if (blocks > sm_count() * 4) blocks = sm_count() * 4;
    k_digit_hist<<<blocks, 256, 0, s>>>(keys_in, num_keys, ctl);
    launch_onesweep32(keys_in, nullptr, keys_b, vals_b, num_keys, 0, ctl, lookback, s);
    launch_onesweep32(keys_b, vals_b, keys_out, perm_out, num_keys, 1, ctl, lookback, s);
    launch_onesweep32(keys_out, perm_out, keys_b, vals_b, num_keys, 2, ctl, lookback, s);
    launch_onesweep32(keys_b, vals_b, keys_out, perm_out, num_keys, 3, ctl, lookback, s);
    if (cudaGetLastError() != cudaSuccess) return LVBH_ECUDA;
    uint32_t err = 0;
    if (cudaMemcpyAsync(&err, &ctl->err, sizeof err, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return LVBH_ECUDA;
    }
    // a look-back wait that gave up, or any other device-side error (a scatter target out of
    // range: keys_out / perm_out are then incomplete)
    if (err & ERR_LOOKBACK_TIMEOUT) return LVBH_ETIMEOUT;
    return err ? LVBH_EDEVICE : LVBH_OK;
}
