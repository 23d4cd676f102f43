// obj.cu - OBJ text -> the build's 48-byte triangle soup and MODEL_BOUNDS, on the device.
//
// Replaces parseObj(file) (scripts/obj/parse-obj.js:3-88) and the OBJFile parser it calls
// (scripts/obj/obj-file-parser.js:19-193), which the demo runs on the main thread before every
// build (main.js:72-73).  The text is parsed in parallel, one thread per line, with the
// reference's semantics:
//   * lines split on '\n' and cut at the first '#'; tokens separated by runs of JavaScript
//     whitespace (`\s`: ASCII \t \n \v \f \r and space, and the UTF-8 forms of U+00A0, U+1680,
//     U+2000-200A, U+2028, U+2029, U+202F, U+205F, U+3000, U+FEFF); keyword lower-cased;
//   * the statements the parser checks fail the parse where the reference throws: g and s with
//     other than one argument (:101-105, :196-201), l with fewer than two vertices or a vertex
//     of more than two '/'-parts (:132-151), f with fewer than three vertices, a vertex of more
//     than three parts or a vertex index parseInt()s to 0 (:153-186);
//   * only model 0 counts (parse-obj.js:17-60): the default model when a v / vt / vn / l / f
//     statement precedes the first `o` (_currentModel, :82-91), else the model the first `o`
//     opens; negative face indices count back from that model's vertices so far, and every
//     index must name one of its vertices (else the reference's array read throws);
//   * vertices are parsed as JavaScript's parseFloat does (longest decimal prefix, correctly
//     rounded), exactly on the device for every decimal exponent within 10^+-27 (see
//     dec_to_double); the rare rest is re-parsed on the host by the C library's correctly
//     rounded strtod;
//   * faces are fan-triangulated from their first vertex, y and z swapped, stored as float32
//     (round to nearest even, the Float32Array of build-bvh.js:14-21), pad 3.1415; bounds are
//     Math.min / Math.max over the faces' vertices in double (NaN absorbs, -0 below +0) from
//     +-1e30, and two floor triangles lie at z_min + .01 (parse-obj.js:62-76).
// Passes: newlines per 4 KB chunk -> scan -> line starts; per-line classify and check; the
// model-0 line range; a 64-bit scan of (vertex count | triangle count) over it; vertices;
// faces -> soup + bounds.  Each pass streams the text from HBM once; its bound is HBM.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lvbh.h"
#include "lvbh_internal.h"

namespace lvbh {

namespace {

typedef unsigned __int128 u128;

constexpr int kT = 256;
constexpr int kChunk = kT * 64;  // text bytes per newline-count block (64 per thread)
constexpr int kScanItems = 16;
constexpr int kScanTile = kT * kScanItems;
constexpr uint32_t kNone = 0xFFFFFFFFu;

enum : uint8_t { LT_NONE = 0, LT_O, LT_G, LT_V, LT_VT, LT_VN, LT_L, LT_S, LT_F };

// Device state of one parse (set to its initial values by the host before the passes).
struct ObjCtl {
    uint32_t err_line;    // smallest 0-based line whose statement throws (kNone: none)
    uint32_t first_o;     // first `o` line (kNone: none)
    uint32_t second_o;    // the next `o` line after it
    uint32_t first_need;  // first v / vt / vn / l / f line (creates the default model)
    uint32_t bad_index;   // a model-0 face names no vertex
    uint32_t num_hard;    // vertex lines left to the host parser
    uint32_t newlines;
    uint32_t m0a, m0b;    // model 0's lines [m0a, m0b)
    uint32_t no_model;    // the text defines no model (output.models[0] is undefined)
    uint32_t pad;
    unsigned long long totals;  // model-0 vertices (low 32 bits) and triangles (high 32 bits)
    unsigned long long bmin[3], bmax[3];  // ordered doubles (ord64)
    uint32_t nan_min[3], nan_max[3];
};

// A vertex line the device leaves to the host: its text [start, end) (up to its comment, or
// further when the device stopped reading before it) and vertex rank.  The same
// slot then carries the host's exact coordinates back (HardFix).
struct HardLine {
    unsigned long long start, end;
    uint32_t vi, pad0;
    uint32_t pad1, pad2;
};
struct HardFix {
    double xyz[3];
    uint32_t vi, pad;
};
static_assert(sizeof(HardLine) == sizeof(HardFix), "hard-line slot");

// Length in bytes of the JavaScript whitespace character at s[i] (0: none), the line ending
// at e.  A UTF-8 lead byte always starts a new character for the decoder of readAsText (an
// unfinished sequence before it becomes U+FFFD), so checking every byte position finds exactly
// the whitespace characters the decoded string holds.
template <typename S>
__host__ __device__ __forceinline__ int ws_len(const S &s, uint64_t i, uint64_t e) {
    const uint8_t c = s[i];
    if (c == ' ' || (c >= 9 && c <= 13)) return 1;
    if (c < 0xC2) return 0;
    if (c == 0xC2) return (i + 1 < e && s[i + 1] == 0xA0) ? 2 : 0;
    if (i + 2 >= e) return 0;
    const uint8_t c1 = s[i + 1], c2 = s[i + 2];
    switch (c) {
        case 0xE1: return (c1 == 0x9A && c2 == 0x80) ? 3 : 0;
        case 0xE2:
            if (c1 == 0x80) return ((c2 >= 0x80 && c2 <= 0x8A) || c2 == 0xA8 || c2 == 0xA9 || c2 == 0xAF) ? 3 : 0;
            return (c1 == 0x81 && c2 == 0x9F) ? 3 : 0;
        case 0xE3: return (c1 == 0x80 && c2 == 0x80) ? 3 : 0;
        case 0xEF: return (c1 == 0xBB && c2 == 0xBF) ? 3 : 0;
    }
    return 0;
}

// Next token of s[i, e): false when none is left; else [a, b).
template <typename S>
__host__ __device__ __forceinline__ bool next_token(const S &s, uint64_t &i, uint64_t e, uint64_t &a,
                                                    uint64_t &b) {
    while (i < e) {
        const int w = ws_len(s, i, e);
        if (!w) break;
        i += w;
    }
    if (i >= e) return false;
    a = i;
    while (i < e && !ws_len(s, i, e)) ++i;
    b = i;
    return true;
}

// Order-preserving map of doubles (-0 below +0) for 64-bit atomic min / max.
__device__ __forceinline__ unsigned long long ord64(double d) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__constant__ double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,
                                  1e8,  1e9,  1e10, 1e11, 1e12, 1e13, 1e14, 1e15,
                                  1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

__device__ __forceinline__ int bitlen128(u128 x) {
    const unsigned long long hi = (unsigned long long)(x >> 64), lo = (unsigned long long)x;
    return hi ? 128 - __clzll((long long)hi) : 64 - __clzll((long long)lo);
}

// (x + f) * 2^e2 rounded to the nearest double, ties to even; x has more than 53 bits or
// f == 0, f in [0, 1) is represented by `sticky` = (f != 0).  The result is a normal double.
__device__ double round_scaled(u128 x, int e2, bool sticky) {
    const int nb = bitlen128(x);
    unsigned long long mant;
    int shift = 0;
    if (nb <= 53) {
        mant = (unsigned long long)x;
    } else {
        shift = nb - 53;
        mant = (unsigned long long)(x >> shift);
        const u128 rem = x & (((u128)1 << shift) - 1), half = (u128)1 << (shift - 1);
        if (rem > half || (rem == half && (sticky || (mant & 1)))) ++mant;
        if (mant == (1ull << 53)) { mant >>= 1; ++shift; }
    }
    const double p2 = __longlong_as_double((long long)(e2 + shift + 1023) << 52);
    return __dmul_rn(__ull2double_rn(mant), p2);  // both exact
}

// w * 10^q correctly rounded (w >= 1): false when q lies outside the device's exact range.
// |q| <= 22 with w <= 2^53 is one IEEE multiply or divide of exact doubles (Clinger, "How to
// read floating point numbers accurately", 1990).  Otherwise, for |q| <= 27 (5^27 < 2^63): the
// exact integer w * 5^q scaled by 2^q, or the 128-bit quotient (w * 2^(64 + lz)) / 5^-q with
// its remainder as the sticky bit, rounded once.
__device__ bool dec_to_double(unsigned long long w, int q, double &out) {
    if (w <= (1ull << 53) && q >= -22 && q <= 22) {
        out = q >= 0 ? __dmul_rn((double)w, kPow10[q]) : __ddiv_rn((double)w, kPow10[-q]);
        return true;
    }
    if (q < -27 || q > 27) return false;
    unsigned long long p5 = 1;
    for (int k = 0; k < (q >= 0 ? q : -q); ++k) p5 *= 5;
    if (q >= 0) {
        out = round_scaled((u128)w * p5, q, false);
        return true;
    }
    const int lz = __clzll((long long)w);
    const u128 n = (u128)(w << lz) << 64;
    const u128 quo = n / p5;
    const u128 rem = n - quo * p5;
    out = round_scaled(quo, q - 64 - lz, rem != 0);  // 2^-(64 + lz) * 2^q * 5^q = 10^q / 2^(64+lz)
    return true;
}

// ---- Line scanning on the device.  A line is b[0, e): b is its first byte in a block's
// shared-memory window or in global memory (each kernel inlines the scan once per case, so the
// window case compiles to shared-memory loads), positions are 32-bit, and the first '#' ends the
// line (cut when the scan reaches it).

// Bytes of the JavaScript whitespace character at b[i] (0: none).
__device__ __forceinline__ uint32_t ws32(const uint8_t *b, uint32_t i, uint32_t e) {
    const uint32_t c = b[i];
    if (c <= 32) return (c == 32 || c - 9u <= 4u) ? 1u : 0u;
    if (c < 0xC2) return 0;
    return (uint32_t)ws_len(b, (uint64_t)i, (uint64_t)e);  // the multi-byte forms
}

// Skips whitespace from i: false at the end of the content (the line's end, or a '#', which
// then becomes the end).
__device__ __forceinline__ bool skip_ws(const uint8_t *b, uint32_t &i, uint32_t &e) {
    while (i < e) {
        if (b[i] == '#') {
            e = i;
            return false;
        }
        const uint32_t w = ws32(b, i, e);
        if (!w) return true;
        i += w;
    }
    return false;
}

// Moves i to the end of the token it is in (whitespace, '#' or the end); returns the number of
// '/' bytes passed.
__device__ __forceinline__ uint32_t skip_token(const uint8_t *b, uint32_t &i, uint32_t &e) {
    uint32_t slashes = 0;
    while (i < e) {
        const uint32_t c = b[i];
        if (c == '#') {
            e = i;
            break;
        }
        if ((c <= 32 || c >= 0xC2) && ws32(b, i, e)) break;
        slashes += c == '/';
        ++i;
    }
    return slashes;
}

constexpr long long kIdxNaN = -0x7FFFFFFFFFFFFFFFll - 1;  // parseInt found no digit
constexpr long long kIdxHuge = kIdxNaN + 1;               // |value| >= 2^53: names no vertex

// parseInt (radix undefined) from b[i]: sign, optional 0x / 0X, the longest digit run (what
// parseInt makes of a face vertex's first '/'-part, which ends where the digits do); i is left
// after the digits.  Values of 2^53 and more name no vertex and are not 0, so they collapse to
// kIdxHuge.
__device__ __forceinline__ long long parse_index(const uint8_t *b, uint32_t &i, uint32_t e) {
    bool neg = false;
    if (i < e && (b[i] == '+' || b[i] == '-')) {
        neg = b[i] == '-';
        ++i;
    }
    uint32_t radix = 10;
    if (i + 1 < e && b[i] == '0' && (b[i + 1] | 0x20u) == 'x') {
        radix = 16;
        i += 2;
    }
    unsigned long long v = 0;
    uint32_t digits = 0;
    while (i < e) {
        const uint32_t c = b[i];
        uint32_t d;
        if (c - '0' <= 9u) d = c - '0';
        else if (radix == 16 && (c | 0x20u) - 'a' <= 5u) d = (c | 0x20u) - 'a' + 10;
        else break;
        v = v < (1ull << 53) ? v * radix + d : v;
        ++digits;
        ++i;
    }
    if (!digits) return kIdxNaN;
    if (v >= (1ull << 53)) return kIdxHuge;
    return neg ? -(long long)v : (long long)v;
}

__constant__ uint32_t kPow10u[10] = {1u, 10u, 100u, 1000u, 10000u, 100000u, 1000000u, 10000000u,
                                     100000000u, 1000000000u};

// parseFloat from b[i], a token's first byte: true with the double in out, false when the host
// parses it (decimal exponent beyond +-27, or more than 19 significant digits whose dropped
// tail could change the rounding); i is left where the literal ends.  Significant digits
// accumulate nine at a time in 32 bits.
__device__ __forceinline__ bool parse_number(const uint8_t *b, uint32_t &i, uint32_t e, double &out) {
    bool neg = false;
    if (i < e && (b[i] == '+' || b[i] == '-')) {
        neg = b[i] == '-';
        ++i;
    }
    if (i + 8 <= e && b[i] == 'I' && b[i + 1] == 'n' && b[i + 2] == 'f' && b[i + 3] == 'i' &&
        b[i + 4] == 'n' && b[i + 5] == 'i' && b[i + 6] == 't' && b[i + 7] == 'y') {
        i += 8;
        out = neg ? -INFINITY : INFINITY;
        return true;
    }
    unsigned long long m = 0;  // folded significant digits
    uint32_t acc = 0, na = 0;  // digits not folded yet (at most 9)
    uint32_t nd = 0;           // significant digits kept (at most 19)
    long long dexp = 0;
    bool any = false, inexact = false, frac = false;
    while (i < e) {
        const uint32_t c = b[i];
        const uint32_t d = c - '0';
        if (d > 9u) {
            if (c == '.' && !frac) {
                frac = true;
                ++i;
                continue;
            }
            break;
        }
        any = true;
        if (nd < 19) {
            if (nd | d) {
                acc = acc * 10 + d;
                ++nd;
                if (++na == 9) {
                    m = m * 1000000000ull + acc;
                    acc = 0;
                    na = 0;
                }
            }
            dexp -= frac;
        } else {
            dexp += !frac;
            inexact |= d != 0;
        }
        ++i;
    }
    if (!any) {
        out = NAN;
        return true;
    }
    m = m * kPow10u[na] + acc;
    long long e10 = 0;
    if (i < e && (b[i] | 0x20u) == 'e') {
        uint32_t j = i + 1;
        bool eneg = false;
        if (j < e && (b[j] == '+' || b[j] == '-')) {
            eneg = b[j] == '-';
            ++j;
        }
        long long ev = 0;
        uint32_t ed = 0;
        while (j < e && b[j] - '0' <= 9u) {
            if (ev < 1000000000ll) ev = ev * 10 + (b[j] - '0');
            ++j;
            ++ed;
        }
        if (ed) {
            e10 = eneg ? -ev : ev;
            i = j;
        }
    }
    if (m == 0) {
        out = neg ? -0.0 : 0.0;
        return true;
    }
    const long long q = e10 + dexp;
    if (q < -27 || q > 27) return false;
    double v;
    if (!dec_to_double(m, (int)q, v)) return false;
    if (inexact) {  // the value lies strictly between m * 10^q and (m + 1) * 10^q
        double hi;
        if (!dec_to_double(m + 1, (int)q, hi) || hi != v) return false;
    }
    out = neg ? -v : v;
    return true;
}

// Line l: its bytes [p, q) (without the '\n').
__device__ __forceinline__ void line_bytes(uint64_t n, const uint64_t *line_start, uint32_t L, uint32_t l,
                                           uint64_t &p, uint64_t &q) {
    p = line_start[l];
    q = l + 1 < L ? line_start[l + 1] - 1 : n;
}

constexpr int kLineBlock = 256;     // lines per block of the per-line kernels
constexpr int kWindow = 24 * 1024;  // text bytes a block stages in shared memory

// Stages the text of lines [l0, l0 + cnt) into win (as much as fits, from the 16-byte boundary
// at or below the first line's start) with coalesced 16-byte loads; [w0, w1) is what it holds.
// Every thread of the block calls it.
__device__ void stage_lines(const uint8_t *__restrict__ text, uint64_t n, const uint64_t *__restrict__ line_start,
                            uint32_t L, uint32_t l0, uint32_t cnt, uint8_t *win, uint64_t &w0, uint64_t &w1) {
    const uint64_t a = line_start[l0] & ~15ull;
    const uint64_t z = l0 + cnt < L ? line_start[l0 + cnt] : n;
    const uint64_t e = z < a + kWindow ? z : a + kWindow;
    for (uint64_t c = a + 16ull * threadIdx.x; c < e; c += 16ull * blockDim.x) {
        if (c + 16 <= n) {
            *reinterpret_cast<uint4 *>(win + (c - a)) = __ldcs(reinterpret_cast<const uint4 *>(text + c));
        } else {
            for (int k = 0; k < 16; ++k)
                if (c + k < n) win[c - a + k] = text[c + k];
        }
    }
    w0 = a;
    w1 = e;
    __syncthreads();
}

__device__ __forceinline__ uint8_t lower(uint8_t c) { return (c >= 'A' && c <= 'Z') ? c + 32 : c; }

__device__ __forceinline__ uint8_t keyword(const uint8_t *b, uint32_t a, uint32_t z) {
    const uint32_t n = z - a;
    if (n == 1) {
        switch (lower(b[a])) {
            case 'o': return LT_O;
            case 'g': return LT_G;
            case 'v': return LT_V;
            case 'l': return LT_L;
            case 's': return LT_S;
            case 'f': return LT_F;
        }
    } else if (n == 2 && lower(b[a]) == 'v') {
        if (lower(b[a + 1]) == 't') return LT_VT;
        if (lower(b[a + 1]) == 'n') return LT_VN;
    }
    return LT_NONE;
}

// Exclusive scan of one value per thread across the block (blockDim.x a multiple of 32).
template <typename U>
__device__ __forceinline__ U block_scan(U x, U *s_warp, U *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    U incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const U y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    U off = 0, all = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
        off += i < warp ? s_warp[i] : (U)0;
        all += s_warp[i];
    }
    __syncthreads();
    if (total) *total = all;
    return off + incl - x;
}

// Smallest value over the warp into *dst (atomically), skipping kNone and values that cannot
// lower it, so that one word shared by the grid sees few atomics.
__device__ __forceinline__ void warp_min_into(uint32_t v, uint32_t *dst) {
    v = __reduce_min_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31) == 0 && v != kNone && v < *(volatile uint32_t *)dst) atomicMin(dst, v);
}

// The 64 text bytes of thread threadIdx.x of chunk blockIdx.x (zero past the end): four
// 16-byte loads; newline count by a SWAR zero-byte test on each word.
__device__ __forceinline__ void load64(const uint8_t *__restrict__ s, uint64_t n, uint64_t p, uint4 (&v)[4]) {
    if (p + 64 <= n) {
#pragma unroll
        for (int j = 0; j < 4; ++j) v[j] = __ldcs(reinterpret_cast<const uint4 *>(s + p) + j);
    } else {
        uint8_t *b = reinterpret_cast<uint8_t *>(v);
        for (int k = 0; k < 64; ++k) b[k] = p + k < n ? s[p + k] : 0;
    }
}

__device__ __forceinline__ uint32_t newlines_in(uint32_t w) {
    const uint32_t x = w ^ 0x0A0A0A0Au;  // zero bytes where '\n' was
    return __popc(~(((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x | 0x7F7F7F7Fu));
}

__device__ __forceinline__ uint32_t newlines64(const uint4 (&v)[4]) {
    uint32_t c = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) c += newlines_in(v[j].x) + newlines_in(v[j].y) + newlines_in(v[j].z) + newlines_in(v[j].w);
    return c;
}

// Newlines per kChunk bytes (64 per thread).
__global__ void __launch_bounds__(kT) k_nl_count(const uint8_t *__restrict__ s, uint64_t n,
                                                 uint32_t *__restrict__ cnt) {
    __shared__ uint32_t w[kT / 32];
    uint4 v[4];
    load64(s, n, (uint64_t)blockIdx.x * kChunk + threadIdx.x * 64ull, v);
    const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, newlines64(v));
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int i = 0; i < kT / 32; ++i) t += w[i];
        cnt[blockIdx.x] = t;
    }
}

// Exclusive scan of v[0, n) in place by one block, each thread over a run of consecutive
// entries; *total = the sum.
template <typename U>
__global__ void __launch_bounds__(1024) k_scan_small(U *v, uint32_t n, U *total) {
    __shared__ U s_warp[32];
    const uint32_t per = (n + 1023) / 1024, b = threadIdx.x * per, e = min(n, b + per);
    U sum = 0;
    for (uint32_t i = b; i < e; ++i) sum += v[i];
    U all;
    U run = block_scan<U>(sum, s_warp, &all);
    for (uint32_t i = b; i < e; ++i) {
        const U x = v[i];
        v[i] = run;
        run += x;
    }
    if (threadIdx.x == 0) *total = all;
}

// Line starts: the newline at byte k (rank r over the text) starts line r + 1 at k + 1.
__global__ void __launch_bounds__(kT) k_nl_write(const uint8_t *__restrict__ s, uint64_t n,
                                                 const uint32_t *__restrict__ base,
                                                 uint64_t *__restrict__ line_start) {
    __shared__ uint32_t s_warp[kT / 32];
    const uint64_t p = (uint64_t)blockIdx.x * kChunk + threadIdx.x * 64ull;
    uint4 v[4];
    load64(s, n, p, v);
    uint32_t r = base[blockIdx.x] + block_scan<uint32_t>(newlines64(v), s_warp, nullptr);
    const uint32_t *w = reinterpret_cast<const uint32_t *>(v);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t m = ~(((w[j] ^ 0x0A0A0A0Au) & 0x7F7F7F7Fu) + 0x7F7F7F7Fu | (w[j] ^ 0x0A0A0A0Au) | 0x7F7F7F7Fu);
        while (m) {  // one bit (7, 15, 23 or 31) per newline byte, in text order
            const int byte = (__ffs(m) - 1) >> 3;
            line_start[++r] = p + 4 * j + byte + 1;
            m &= m - 1;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) line_start[0] = 0;
}

struct LineClass {
    uint8_t type;
    bool bad;
    uint32_t fan;
};

// Statement type of the line b[0, len), whether the reference's parser throws on it (g / s
// with other than one argument, l with fewer than two vertices or a vertex of more than two
// '/'-parts, f with fewer than three vertices, a vertex of more than three parts or a first
// part parseInt()s to 0 or -0), and the triangles a face fans into.
__device__ __forceinline__ LineClass classify(const uint8_t *b, uint32_t len) {
    uint32_t i = 0, e = len;
    if (!skip_ws(b, i, e)) return {LT_NONE, false, 0};
    const uint32_t a = i;
    skip_token(b, i, e);
    const uint8_t t = keyword(b, a, i);
    if (t == LT_NONE) return {LT_NONE, false, 0};
    uint32_t ntok = 1;
    bool bad = false;
    while (skip_ws(b, i, e)) {
        ++ntok;
        if (t == LT_F) {
            bad |= parse_index(b, i, e) == 0;
            bad |= skip_token(b, i, e) > 2;
        } else if (t == LT_L) {
            bad |= skip_token(b, i, e) > 1;
        } else {
            skip_token(b, i, e);
        }
    }
    if ((t == LT_G || t == LT_S) && ntok != 2) bad = true;
    if (t == LT_L && ntok < 3) bad = true;
    uint32_t fan = 0;
    if (t == LT_F) {
        if (ntok < 4) bad = true;
        else fan = ntok - 3;
    }
    return {t, bad, fan};
}

// Per line: its class, and the first `o` and model-creating lines.  One block per kLineBlock
// lines, their text staged in shared memory.
__global__ void __launch_bounds__(kLineBlock) k_lines(const uint8_t *__restrict__ text, uint64_t n,
                                                      const uint64_t *__restrict__ line_start, uint32_t L,
                                                      uint8_t *__restrict__ type, uint32_t *__restrict__ fans,
                                                      ObjCtl *__restrict__ ctl) {
    __shared__ __align__(16) uint8_t win[kWindow];
    const uint32_t l0 = blockIdx.x * kLineBlock, l = l0 + threadIdx.x;
    uint64_t w0, w1;
    stage_lines(text, n, line_start, L, l0, min((uint32_t)kLineBlock, L - l0), win, w0, w1);
    LineClass c{LT_NONE, false, 0};
    if (l < L) {
        uint64_t p, q;
        line_bytes(n, line_start, L, l, p, q);
        if (p >= w0 && q <= w1) c = classify(win + (p - w0), (uint32_t)(q - p));
        else c = classify(text + p, (uint32_t)(q - p));
        type[l] = c.type;
        fans[l] = c.fan;
    }
    warp_min_into(c.bad ? l : kNone, &ctl->err_line);
    warp_min_into(c.type == LT_O ? l : kNone, &ctl->first_o);
    const bool need = c.type == LT_V || c.type == LT_VT || c.type == LT_VN || c.type == LT_L || c.type == LT_F;
    warp_min_into(need ? l : kNone, &ctl->first_need);
}

// The first `o` line after the first one.
__global__ void __launch_bounds__(kT) k_second_o(const uint8_t *__restrict__ type, uint32_t L,
                                                 ObjCtl *__restrict__ ctl) {
    const uint32_t fo = ctl->first_o;
    if (fo == kNone) return;
    const uint32_t l = blockIdx.x * kT + threadIdx.x;
    warp_min_into(l < L && l > fo && type[l] == LT_O ? l : kNone, &ctl->second_o);
}

// Model 0's lines: the default model when a model-creating statement precedes the first `o`
// (_currentModel, obj-file-parser.js:82-91), else the model that `o` opens, up to the next `o`.
__global__ void k_model_range(uint32_t L, ObjCtl *__restrict__ ctl) {
    const uint32_t fo = ctl->first_o, fn = ctl->first_need, so = ctl->second_o;
    uint32_t a = 0, b = 0, none = 0;
    if (fn != kNone && (fo == kNone || fn < fo)) {
        b = fo == kNone ? L : fo;
    } else if (fo != kNone) {
        a = fo;
        b = so == kNone ? L : so;
    } else {
        none = 1;
    }
    ctl->m0a = a;
    ctl->m0b = b;
    ctl->no_model = none;
}

// Packed count of a model-0 line: one vertex (low 32 bits) or a face's triangles (high).
__device__ __forceinline__ unsigned long long line_count(const uint8_t *type, const uint32_t *fans,
                                                         uint32_t l) {
    const uint8_t t = type[l];
    return t == LT_V ? 1ull : t == LT_F ? (unsigned long long)fans[l] << 32 : 0ull;
}

// Tile sums of the packed counts of the L lines (zero outside model 0's [m0a, m0b)).
__global__ void __launch_bounds__(kT) k_scan_up(const uint8_t *__restrict__ type,
                                                const uint32_t *__restrict__ fans, uint32_t L,
                                                const ObjCtl *__restrict__ ctl,
                                                unsigned long long *__restrict__ sums) {
    __shared__ unsigned long long s_warp[kT / 32];
    const uint32_t a = ctl->m0a, b = ctl->m0b;
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    unsigned long long t = 0;
    for (int k = 0; k < kScanItems; ++k)
        if (base + k >= a && base + k < b) t += line_count(type, fans, (uint32_t)(base + k));
    unsigned long long all;
    block_scan<unsigned long long>(t, s_warp, &all);
    if (threadIdx.x == 0) sums[blockIdx.x] = all;
}

// pre[l]: exclusive prefix of the packed counts at line l.
__global__ void __launch_bounds__(kT) k_scan_down(const uint8_t *__restrict__ type,
                                                  const uint32_t *__restrict__ fans, uint32_t L,
                                                  const ObjCtl *__restrict__ ctl,
                                                  const unsigned long long *__restrict__ sums,
                                                  unsigned long long *__restrict__ pre) {
    __shared__ unsigned long long s_warp[kT / 32];
    const uint32_t a = ctl->m0a, b = ctl->m0b;
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    unsigned long long x[kScanItems], t = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        x[k] = (base + k >= a && base + k < b) ? line_count(type, fans, (uint32_t)(base + k)) : 0ull;
        t += x[k];
    }
    unsigned long long run = sums[blockIdx.x] + block_scan<unsigned long long>(t, s_warp, nullptr);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < L) pre[base + k] = run;
        run += x[k];
    }
}

struct VertexParse {
    double x, y, z;
    uint32_t end;  // where the scan stopped (the content's end when a number was left over)
    bool ok;
};

// The coordinates of the vertex line b[0, len) (missing ones 0, as _parseVertexCoords has it).
__device__ __forceinline__ VertexParse parse_vertex(const uint8_t *b, uint32_t len) {
    VertexParse r{0.0, 0.0, 0.0, len, true};
    uint32_t i = 0, e = len;
    skip_ws(b, i, e);
    skip_token(b, i, e);  // the keyword
    if (skip_ws(b, i, e)) {
        r.ok &= parse_number(b, i, e, r.x);
        skip_token(b, i, e);
        if (skip_ws(b, i, e)) {
            r.ok &= parse_number(b, i, e, r.y);
            skip_token(b, i, e);
            if (skip_ws(b, i, e)) {
                r.ok &= parse_number(b, i, e, r.z);
                skip_token(b, i, e);
            }
        }
    }
    r.end = e;
    return r;
}

// Model-0 vertex lines -> doubles at their rank; numbers outside the device's exact range are
// listed for the host.  One block per kLineBlock lines of model 0, its text staged when it holds
// a vertex line.
__global__ void __launch_bounds__(kLineBlock) k_vertices(const uint8_t *__restrict__ text, uint64_t n,
                                                         const uint64_t *__restrict__ line_start, uint32_t L,
                                                         const uint8_t *__restrict__ type, uint32_t a, uint32_t m,
                                                         const unsigned long long *__restrict__ pre,
                                                         double *__restrict__ verts, HardLine *__restrict__ hard,
                                                         ObjCtl *__restrict__ ctl) {
    __shared__ __align__(16) uint8_t win[kWindow];
    const uint32_t i0 = blockIdx.x * kLineBlock, i = i0 + threadIdx.x;
    const bool mine = i < m && type[a + i] == LT_V;
    if (!__syncthreads_or(mine)) return;
    uint64_t w0, w1;
    stage_lines(text, n, line_start, L, a + i0, min((uint32_t)kLineBlock, m - i0), win, w0, w1);
    if (!mine) return;
    uint64_t p, q;
    line_bytes(n, line_start, L, a + i, p, q);
    VertexParse r;
    if (p >= w0 && q <= w1) r = parse_vertex(win + (p - w0), (uint32_t)(q - p));
    else r = parse_vertex(text + p, (uint32_t)(q - p));
    const uint32_t vi = (uint32_t)(pre[a + i] & 0xFFFFFFFFull);
    verts[3ull * vi] = r.x;
    verts[3ull * vi + 1] = r.y;
    verts[3ull * vi + 2] = r.z;
    if (!r.ok) {
        const uint32_t h = atomicAdd(&ctl->num_hard, 1u);
        hard[h] = HardLine{p, p + r.end, vi, 0u, 0u, 0u};
    }
}

__global__ void __launch_bounds__(kT) k_patch(const HardFix *__restrict__ fix, uint32_t count,
                                              double *__restrict__ verts) {
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i >= count) return;
    const HardFix f = fix[i];
    verts[3ull * f.vi] = f.xyz[0];
    verts[3ull * f.vi + 1] = f.xyz[1];
    verts[3ull * f.vi + 2] = f.xyz[2];
}

// float32 of a coordinate as Float32Array stores it (NaN as the quiet NaN 0x7FC00000).
__device__ __forceinline__ float to_f32(double d) {
    return isnan(d) ? __int_as_float(0x7FC00000) : __double2float_rn(d);
}

// Running Math.min / Math.max of one thread's vertices (ordered doubles, NaN flags).
struct BoundsAcc {
    unsigned long long mn[3], mx[3];
    bool nan[3];
    __device__ __forceinline__ void add(const double (&c)[3]) {
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            if (isnan(c[ax])) {
                nan[ax] = true;
                continue;
            }
            const unsigned long long o = ord64(c[ax]);
            mn[ax] = o < mn[ax] ? o : mn[ax];
            mx[ax] = o > mx[ax] ? o : mx[ax];
        }
    }
};

// The face line b[0, len): its vertices resolved (negative indices against `before`, the
// model's vertices so far), fanned from the first, stored from triangle `out` on; false when an
// index names no vertex.
__device__ __forceinline__ bool emit_face(const uint8_t *b, uint32_t len, long long before, uint32_t nverts,
                                          const double *__restrict__ verts, float4 *__restrict__ tri,
                                          unsigned long long out, BoundsAcc &bd) {
    uint32_t i = 0, e = len;
    skip_ws(b, i, e);
    skip_token(b, i, e);  // the keyword
    const float pad = __double2float_rn(3.1415);
    float4 r = make_float4(0.f, 0.f, 0.f, pad), prev = r;
    int nv = 0;
    while (skip_ws(b, i, e)) {
        long long v = parse_index(b, i, e);
        skip_token(b, i, e);
        if (v == kIdxNaN || v == kIdxHuge) return false;
        if (v < 0) v = before + 1 + v;  // vertices.length + 1 + vertexIndex
        const long long vk = v - 1;
        if (vk < 0 || vk >= (long long)nverts) return false;
        const double *vp = verts + 3ull * (unsigned long long)vk;
        const double c[3] = {vp[0], vp[2], vp[1]};  // x, then the file's z as y and y as z
        bd.add(c);
        const float4 cur = make_float4(to_f32(c[0]), to_f32(c[1]), to_f32(c[2]), pad);
        if (nv == 0) {
            r = cur;
        } else if (nv >= 2) {
            float4 *o = tri + 3ull * out;
            o[0] = r;
            o[1] = prev;
            o[2] = cur;
            ++out;
        }
        prev = cur;
        ++nv;
    }
    return true;
}

// Model-0 faces -> fan triangles (y and z swapped, float32, pad 3.1415) and the bounds.  One
// block per kLineBlock lines of model 0, its text staged when it holds a face line.
__global__ void __launch_bounds__(kLineBlock) k_faces(const uint8_t *__restrict__ text, uint64_t n,
                                                      const uint64_t *__restrict__ line_start, uint32_t L,
                                                      const uint8_t *__restrict__ type, uint32_t a, uint32_t m,
                                                      const unsigned long long *__restrict__ pre, uint32_t nverts,
                                                      const double *__restrict__ verts, float4 *__restrict__ tri,
                                                      ObjCtl *__restrict__ ctl) {
    __shared__ __align__(16) uint8_t win[kWindow];
    const uint32_t i0 = blockIdx.x * kLineBlock, i = i0 + threadIdx.x;
    const bool mine = i < m && type[a + i] == LT_F;
    if (!__syncthreads_or(mine)) return;
    uint64_t w0, w1;
    stage_lines(text, n, line_start, L, a + i0, min((uint32_t)kLineBlock, m - i0), win, w0, w1);
    BoundsAcc bd{{~0ull, ~0ull, ~0ull}, {0ull, 0ull, 0ull}, {false, false, false}};
    if (mine) {
        uint64_t p, q;
        line_bytes(n, line_start, L, a + i, p, q);
        const long long before = (long long)(pre[a + i] & 0xFFFFFFFFull);  // model-0 vertices so far
        const unsigned long long out = pre[a + i] >> 32;
        bool ok;
        if (p >= w0 && q <= w1) ok = emit_face(win + (p - w0), (uint32_t)(q - p), before, nverts, verts, tri, out, bd);
        else ok = emit_face(text + p, (uint32_t)(q - p), before, nverts, verts, tri, out, bd);
        if (!ok) atomicOr(&ctl->bad_index, 1u);
    }
    __shared__ unsigned long long s_mn[3][kLineBlock / 32], s_mx[3][kLineBlock / 32];
    __shared__ int s_nan[3][kLineBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        unsigned long long lo = bd.mn[ax], hi = bd.mx[ax];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long lo2 = __shfl_xor_sync(0xFFFFFFFFu, lo, o);
            const unsigned long long hi2 = __shfl_xor_sync(0xFFFFFFFFu, hi, o);
            lo = lo2 < lo ? lo2 : lo;
            hi = hi2 > hi ? hi2 : hi;
        }
        const int nan_any = __any_sync(0xFFFFFFFFu, bd.nan[ax]);
        if (lane == 0) { s_mn[ax][warp] = lo; s_mx[ax][warp] = hi; s_nan[ax][warp] = nan_any; }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        const int ax = threadIdx.x;
        unsigned long long lo = ~0ull, hi = 0ull;
        int nan_any = 0;
        for (int w = 0; w < kLineBlock / 32; ++w) {
            lo = s_mn[ax][w] < lo ? s_mn[ax][w] : lo;
            hi = s_mx[ax][w] > hi ? s_mx[ax][w] : hi;
            nan_any |= s_nan[ax][w];
        }
        if (lo != ~0ull && lo < *(volatile unsigned long long *)&ctl->bmin[ax]) atomicMin(&ctl->bmin[ax], lo);
        if (hi != 0ull && hi > *(volatile unsigned long long *)&ctl->bmax[ax]) atomicMax(&ctl->bmax[ax], hi);
        if (nan_any && !*(volatile uint32_t *)&ctl->nan_min[ax]) {
            atomicOr(&ctl->nan_min[ax], 1u);
            atomicOr(&ctl->nan_max[ax], 1u);
        }
    }
}

// The floor (parse-obj.js:62-76): two triangles at z_min + .01, 10000 out in x and y, after the
// model's triangles; z_min = Math.min from 1e30 over the faces' vertices (NaN absorbs).
__global__ void k_floor(const ObjCtl *__restrict__ ctl, float4 *__restrict__ tri_floor) {
    const int v = threadIdx.x;  // 6 vertices
    if (v >= 6) return;
    double zmin = 1e30;
    if (ctl->nan_min[2]) {
        zmin = NAN;
    } else if (ctl->bmin[2] != ~0ull) {
        const unsigned long long o = ctl->bmin[2];
        const double d = __longlong_as_double((long long)((o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o));
        zmin = d < 1e30 ? d : 1e30;
    }
    const float h = to_f32(__dadd_rn(zmin, .01)), f = 10000.0f, pad = __double2float_rn(3.1415);
    const float xs[6] = {-f, f, -f, f, f, -f}, ys[6] = {-f, -f, f, -f, f, f};
    tri_floor[v] = make_float4(xs[v], ys[v], h, pad);
}

// parseFloat of a whitespace-free token on the host, for the numbers the device leaves to it:
// the C library's correctly rounded strtod on the longest decimal prefix.
double host_parse_float(const uint8_t *t, size_t len) {
    size_t i = 0;
    bool neg = false;
    if (i < len && (t[i] == '+' || t[i] == '-')) { neg = t[i] == '-'; ++i; }
    if (len - i >= 8 && std::memcmp(t + i, "Infinity", 8) == 0) return neg ? -INFINITY : INFINITY;
    const size_t st = i;
    size_t digits = 0;
    while (i < len && t[i] >= '0' && t[i] <= '9') { ++i; ++digits; }
    if (i < len && t[i] == '.') {
        ++i;
        while (i < len && t[i] >= '0' && t[i] <= '9') { ++i; ++digits; }
    }
    if (!digits) return NAN;
    size_t end = i;
    if (i < len && (t[i] == 'e' || t[i] == 'E')) {
        size_t j = i + 1;
        if (j < len && (t[j] == '+' || t[j] == '-')) ++j;
        size_t ed = 0;
        while (j < len && t[j] >= '0' && t[j] <= '9') { ++j; ++ed; }
        if (ed) end = j;
    }
    const std::string lit(reinterpret_cast<const char *>(t) + st, end - st);
    const double v = std::strtod(lit.c_str(), nullptr);
    return neg ? -v : v;
}

double ord64_inv(unsigned long long o) {
    const unsigned long long u = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
    double d;
    std::memcpy(&d, &u, 8);
    return d;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Grow one scratch block to at least `need` bytes (contents are not kept).
cudaError_t grow(void *&p, size_t &have, size_t need) {
    if (need <= have) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    have = 0;
    const cudaError_t e = cudaMalloc(&p, need);
    if (e == cudaSuccess) have = need;
    return e;
}

}  // namespace

int obj_parse(ObjScratch &sc, const char *text, uint64_t bytes, bool host_text, const float **tri_out,
              uint32_t *num_tris, double *bounds6, uint64_t *err_line, cudaStream_t s,
              std::string &err) {
    auto cuda = [&](cudaError_t e, const char *what) -> int {
        if (e == cudaSuccess) return LVBH_OK;
        cudaGetLastError();
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? LVBH_ENOMEM : LVBH_ECUDA;
    };
#define OBJ_CUDA(call, what)                          \
    do {                                              \
        if (int rc_ = cuda((call), what)) return rc_; \
    } while (0)
    auto reject = [&](uint64_t line, const std::string &msg) {
        *err_line = line;
        err = msg;
        return LVBH_EPARSE;
    };
    *err_line = 0;
    if (!sc.host) OBJ_CUDA(cudaMallocHost(&sc.host, sizeof(ObjCtl)), "cudaMallocHost");
    ObjCtl *hc = static_cast<ObjCtl *>(sc.host);
    // text (staged when it is host memory or not 16-byte aligned), control block, newline
    // counts per chunk
    const uint32_t chunks = (uint32_t)((bytes + kChunk - 1) / kChunk);
    const bool stage = host_text || (reinterpret_cast<uintptr_t>(text) & 15u);
    const size_t text_part = stage ? align256(bytes) : 0;
    OBJ_CUDA(grow(sc.text, sc.text_bytes, text_part + align256(sizeof(ObjCtl)) + align256((chunks + 1) * 4ull)),
             "cudaMalloc(obj text)");
    const uint8_t *d_text = reinterpret_cast<const uint8_t *>(text);
    char *c = static_cast<char *>(sc.text);
    if (stage) {
        if (bytes) OBJ_CUDA(cudaMemcpyAsync(c, text, bytes, host_text ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s),
                            "cudaMemcpyAsync(text)");
        d_text = reinterpret_cast<const uint8_t *>(c);
        c += text_part;
    }
    ObjCtl *ctl = reinterpret_cast<ObjCtl *>(c);
    uint32_t *cnt = reinterpret_cast<uint32_t *>(c + align256(sizeof(ObjCtl)));
    std::memset(hc, 0, sizeof(ObjCtl));
    hc->err_line = hc->first_o = hc->second_o = hc->first_need = kNone;
    for (int a = 0; a < 3; ++a) hc->bmin[a] = ~0ull;
    OBJ_CUDA(cudaMemcpyAsync(ctl, hc, sizeof(ObjCtl), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(ctl)");
    if (chunks) {
        k_nl_count<<<chunks, kT, 0, s>>>(d_text, bytes, cnt);
        k_scan_small<uint32_t><<<1, 1024, 0, s>>>(cnt, chunks, &ctl->newlines);
        OBJ_CUDA(cudaGetLastError(), "k_nl_count");
        OBJ_CUDA(cudaMemcpyAsync(&hc->newlines, &ctl->newlines, 4, cudaMemcpyDeviceToHost, s), "readback");
    }
    OBJ_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const uint32_t L = hc->newlines + 1;
    // per-line arrays: starts, types, fan counts; then (model-0 range only) prefixes
    const size_t lines_need = align256((L + 1ull) * 8) + align256(L) + align256(L * 4ull) +
                              align256(L * 8ull) + align256(((L + (uint64_t)kScanTile - 1) / kScanTile + 1) * 8);
    OBJ_CUDA(grow(sc.lines, sc.lines_bytes, lines_need), "cudaMalloc(obj lines)");
    char *cl = static_cast<char *>(sc.lines);
    uint64_t *line_start = reinterpret_cast<uint64_t *>(cl);
    cl += align256((L + 1ull) * 8);
    uint8_t *type = reinterpret_cast<uint8_t *>(cl);
    cl += align256(L);
    uint32_t *fans = reinterpret_cast<uint32_t *>(cl);
    cl += align256(L * 4ull);
    unsigned long long *pre = reinterpret_cast<unsigned long long *>(cl);
    cl += align256(L * 8ull);
    unsigned long long *sums = reinterpret_cast<unsigned long long *>(cl);
    if (chunks) k_nl_write<<<chunks, kT, 0, s>>>(d_text, bytes, cnt, line_start);
    else OBJ_CUDA(cudaMemsetAsync(line_start, 0, 8, s), "cudaMemsetAsync");
    const uint32_t lb = (uint32_t)((L + (uint64_t)kT - 1) / kT);
    const uint32_t tiles = (uint32_t)((L + (uint64_t)kScanTile - 1) / kScanTile);
    // lines, model 0 and the vertex / triangle prefixes in one stream-ordered run (the first
    // `o`, the model range and the scan read what the kernels before them left in ctl)
    k_lines<<<lb, kLineBlock, 0, s>>>(d_text, bytes, line_start, L, type, fans, ctl);
    k_second_o<<<lb, kT, 0, s>>>(type, L, ctl);
    k_model_range<<<1, 1, 0, s>>>(L, ctl);
    k_scan_up<<<tiles, kT, 0, s>>>(type, fans, L, ctl, sums);
    k_scan_small<unsigned long long><<<1, 1024, 0, s>>>(sums, tiles, &ctl->totals);
    k_scan_down<<<tiles, kT, 0, s>>>(type, fans, L, ctl, sums, pre);
    OBJ_CUDA(cudaGetLastError(), "k_lines");
    OBJ_CUDA(cudaMemcpyAsync(hc, ctl, sizeof(ObjCtl), cudaMemcpyDeviceToHost, s), "readback");
    OBJ_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (hc->err_line != kNone)
        return reject(hc->err_line + 1ull, "line " + std::to_string(hc->err_line + 1ull) +
                                                ": a statement the OBJ parser rejects");
    if (hc->no_model) return reject(0, "the OBJ text defines no model");
    const uint32_t m0a = hc->m0a, m = hc->m0b - hc->m0a;
    const uint32_t mb = (uint32_t)((m + (uint64_t)kLineBlock - 1) / kLineBlock);
    const uint32_t nverts = (uint32_t)(hc->totals & 0xFFFFFFFFull);
    const uint64_t nfan = hc->totals >> 32;
    if (nfan + 2 > LVBH_MAX_TRIS) return reject(0, "the OBJ text makes more than LVBH_MAX_TRIS triangles");
    const uint32_t ntri = (uint32_t)nfan + 2;
    // the soup first (16-byte aligned), then the vertices and the hard-line slots
    const size_t tbytes = align256(ntri * 48ull), vbytes = align256(nverts * 24ull);
    OBJ_CUDA(grow(sc.soup, sc.soup_bytes, tbytes + vbytes + align256(nverts * (size_t)sizeof(HardLine))),
             "cudaMalloc(obj soup)");
    float4 *tri = static_cast<float4 *>(sc.soup);
    double *verts = reinterpret_cast<double *>(static_cast<char *>(sc.soup) + tbytes);
    HardLine *hard = reinterpret_cast<HardLine *>(static_cast<char *>(sc.soup) + tbytes + vbytes);
    // vertices, faces and the floor, then one read-back; numbers the device left to the host
    // (rare) are patched in and the faces and floor run again
    auto faces_and_floor = [&]() {
        if (nfan && mb)
            k_faces<<<mb, kLineBlock, 0, s>>>(d_text, bytes, line_start, L, type, m0a, m, pre, nverts, verts, tri, ctl);
        k_floor<<<1, 32, 0, s>>>(ctl, tri + 3ull * nfan);
    };
    if (nverts && mb)
        k_vertices<<<mb, kLineBlock, 0, s>>>(d_text, bytes, line_start, L, type, m0a, m, pre, verts, hard, ctl);
    faces_and_floor();
    OBJ_CUDA(cudaGetLastError(), "k_faces");
    OBJ_CUDA(cudaMemcpyAsync(hc, ctl, sizeof(ObjCtl), cudaMemcpyDeviceToHost, s), "readback");
    OBJ_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const uint32_t nh = nverts ? hc->num_hard : 0;
    if (nh) {
        std::vector<HardLine> hl(nh);
        OBJ_CUDA(cudaMemcpyAsync(hl.data(), hard, nh * sizeof(HardLine), cudaMemcpyDeviceToHost, s), "readback");
        OBJ_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        std::vector<HardFix> fix(nh);
        std::vector<uint8_t> buf;
        for (uint32_t h = 0; h < nh; ++h) {
            uint64_t len = hl[h].end - hl[h].start;
            const uint8_t *ln = reinterpret_cast<const uint8_t *>(text) + hl[h].start;
            if (!host_text) {
                buf.resize(len);
                if (len) OBJ_CUDA(cudaMemcpy(buf.data(), d_text + hl[h].start, len, cudaMemcpyDeviceToHost), "readback");
                ln = buf.data();
            }
            const void *hash = len ? std::memchr(ln, '#', len) : nullptr;  // the comment cut
            if (hash) len = static_cast<const uint8_t *>(hash) - ln;
            uint64_t k = 0, ta = 0, tb = 0;
            next_token(ln, k, len, ta, tb);  // the keyword
            HardFix f{{0.0, 0.0, 0.0}, hl[h].vi, 0u};
            for (int a = 0; a < 3; ++a) {
                if (!next_token(ln, k, len, ta, tb)) break;
                f.xyz[a] = host_parse_float(ln + ta, tb - ta);
            }
            fix[h] = f;
        }
        HardFix *dfix = reinterpret_cast<HardFix *>(hard);
        OBJ_CUDA(cudaMemcpyAsync(dfix, fix.data(), nh * sizeof(HardFix), cudaMemcpyHostToDevice, s),
                 "cudaMemcpyAsync(fix)");
        k_patch<<<(nh + kT - 1) / kT, kT, 0, s>>>(dfix, nh, verts);
        // the bounds and the index check start over
        for (int a = 0; a < 3; ++a) {
            hc->bmin[a] = ~0ull;
            hc->bmax[a] = 0ull;
            hc->nan_min[a] = hc->nan_max[a] = 0u;
        }
        hc->bad_index = 0u;
        OBJ_CUDA(cudaMemcpyAsync(ctl, hc, sizeof(ObjCtl), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(ctl)");
        faces_and_floor();
        OBJ_CUDA(cudaGetLastError(), "k_faces");
        OBJ_CUDA(cudaMemcpyAsync(hc, ctl, sizeof(ObjCtl), cudaMemcpyDeviceToHost, s), "readback");
        OBJ_CUDA(cudaStreamSynchronize(s), "cudaStreamSynchronize");  // also: `fix` is pageable
    }
    if (hc->bad_index) return reject(0, "a face of model 0 names a vertex the model does not have");
    // bounds: Math.min / Math.max from 1e30 / -1e30 over the faces' vertices
    for (int a = 0; a < 3; ++a) {
        const double lo = hc->bmin[a] == ~0ull ? 1e30 : ord64_inv(hc->bmin[a]);
        const double hi = hc->bmax[a] == 0ull ? -1e30 : ord64_inv(hc->bmax[a]);
        bounds6[a] = hc->nan_min[a] ? NAN : (lo < 1e30 ? lo : 1e30);
        bounds6[3 + a] = hc->nan_max[a] ? NAN : (hi > -1e30 ? hi : -1e30);
    }
    *tri_out = reinterpret_cast<const float *>(tri);
    *num_tris = ntri;
#undef OBJ_CUDA
    return LVBH_OK;
}

void obj_free(ObjScratch &sc) {
    if (sc.text) cudaFree(sc.text);
    if (sc.lines) cudaFree(sc.lines);
    if (sc.soup) cudaFree(sc.soup);
    if (sc.host) cudaFreeHost(sc.host);
    sc = ObjScratch{};
}

}  // namespace lvbh
