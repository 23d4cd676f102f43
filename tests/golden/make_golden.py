"""Generate the golden fixtures in tests/golden/ from a literal simulation of the reference WGSL.

The reference (AddisonPrairie/WebGPU-LVBH-demo) ships no tests, golden vectors or fixtures
and cannot run in this environment (its shaders need a browser WebGPU device).  This script
is the second, independent restatement that pins the C++ oracle: it transliterates each
WGSL entry point line by line, executing workgroups the way the shader text describes them:

  compute_aabb_z_idx     scripts/bvh/kernels/aabb-z-idx.js:177-209 (float32 scalar ops)
  init_idx / init_off    scripts/bvh/kernels/radix-sort.js:526-570 (per-workgroup atomics)
  scan_up                scripts/bvh/kernels/radix-sort.js:763-803
  scan_and_sort          scripts/bvh/kernels/radix-sort.js:575-629
  workgroup_scan         scripts/bvh/kernels/radix-sort.js:653-741, simulated barrier step by
                         barrier step over the 64-entry shared array
  radix tree             scripts/bvh/kernels/radix-tree.js:137-238, including the bit loop of
                         dif() and the split loop that runs until its i32 step overflows
  bvh_upward_pass        scripts/bvh/kernels/bvh-up-pass.js:200-280, every leaf thread a state
                         machine, interleaved by a seeded random scheduler, the 0.0-sentinel
                         spin included, so the arrival order varies as it does on a GPU
  rearrange_triangles    scripts/bvh/kernels/rearrange.js:162-169
  intersect_bvh          scripts/pathtracer/pathtracer.js:495-628 (float32 scalar ops)

The up-pass result is brought to canonical form (Karras left child in the left slot, words 7
and 15 set to 2 and 0) exactly as lvbh.h documents.  Pure Python: sizes stay small.

Usage:  python tests/golden/make_golden.py        (rewrites tests/golden/golden.npz)
"""
from __future__ import annotations

import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "webgpu-lvbh-demo_b200"))

from lvbh import scenes  # noqa: E402

F = np.float32
M32 = 0xFFFFFFFF


# ---------------------------------------------------------------- compute_aabb_z_idx
def u32_of_f32(x: np.float32) -> int:
    """WGSL u32(f32): truncation toward zero, saturating, NaN -> 0."""
    if x != x:
        return 0
    if x <= F(0):
        return 0
    if x >= F(4294967296.0):
        return M32
    return int(x)


def split_3(u: int) -> int:
    x = u & M32
    x = (x | (x << 16)) & 0x030000FF
    x = (x | (x << 8)) & 0x0300F00F
    x = (x | (x << 4)) & 0x030C30C3
    x = (x | (x << 2)) & 0x09249249
    return x


def morton_code(x: int, y: int, z: int) -> int:
    return (split_3(x) | (split_3(y) << 1) | (split_3(z) << 2)) & M32


def wmin(a, b):
    return a if a < b else b


def wmax(a, b):
    return a if a > b else b


def aabb_z_idx(tri: np.ndarray, bounds: np.ndarray):
    n = tri.shape[0]
    aabb = np.zeros((n, 8), dtype=np.float32)
    keys = np.zeros(n, dtype=np.uint32)
    umin = [F(bounds[0]), F(bounds[1]), F(bounds[2])]
    umax = [F(bounds[3]), F(bounds[4]), F(bounds[5])]
    with np.errstate(all="ignore"):
        for i in range(n):
            q = []
            for a in range(3):
                v0, v1, v2 = F(tri[i, a]), F(tri[i, 4 + a]), F(tri[i, 8 + a])
                bmin = wmin(v0, wmin(v1, v2))
                bmax = wmax(v0, wmax(v1, v2))
                aabb[i, a] = bmin
                aabb[i, 4 + a] = bmax
                cen = F(F(bmax + bmin) * F(0.5))
                rel = F(F(cen - umin[a]) / F(umax[a] - umin[a]))
                q.append(u32_of_f32(F(rel * F(1023.99))))
            keys[i] = morton_code(*q)
    return aabb, keys


# ---------------------------------------------------------------- radix sort
def workgroup_scan(scan_arr):
    """The 64-entry up/down-sweep of radix-sort.js:653-741, one barrier phase at a time.
    scan_arr: list of 64 4-lists (vec4u); modified in place."""
    def phase(cond, fn):
        new = [list(v) for v in scan_arr]
        for idx in range(64):
            if cond(idx):
                new[idx] = fn(idx)
        scan_arr[:] = new

    add = lambda a, b: [(x + y) & M32 for x, y in zip(a, b)]  # noqa: E731
    sub = lambda a, b: [(x - y) & M32 for x, y in zip(a, b)]  # noqa: E731
    phase(lambda i: (1 & i) == 1, lambda i: add(scan_arr[i], scan_arr[i - 1]))
    phase(lambda i: (3 & i) == 3, lambda i: add(scan_arr[i], scan_arr[i - 2]))
    phase(lambda i: (7 & i) == 7, lambda i: add(scan_arr[i], scan_arr[i - 4]))
    phase(lambda i: (15 & i) == 15, lambda i: add(scan_arr[i], scan_arr[i - 8]))
    phase(lambda i: (31 & i) == 31, lambda i: add(scan_arr[i], scan_arr[i - 16]))
    phase(lambda i: i == 63, lambda i: list(scan_arr[31]))
    phase(lambda i: i == 31, lambda i: [0, 0, 0, 0])
    for b in (16, 8, 4, 2, 1):
        m = b - 1
        phase(lambda i, m=m, b=b: (m & i) == m and (i & b) != 0,
              lambda i, b=b: add(scan_arr[i], scan_arr[i - b]))
        phase(lambda i, m=m, b=b: (m & i) == m and (i & b) == 0,
              lambda i, b=b: sub(scan_arr[i + b], scan_arr[i]))


def get_val_u32(v: int, win: int) -> int:
    return (v >> (2 * win)) & 3


def get_val_vec(v: int, win: int):
    s = get_val_u32(v, win)
    out = [0, 0, 0, 0]
    out[s] = 1
    return out


def radix_sort(keys: np.ndarray):
    size = keys.size
    vals = [list(int(k) for k in keys), [0] * size]
    idxs = [[0] * size, [0] * size]
    n_wg = (size + 255) // 256
    l1 = [[0, 0, 0, 0] for _ in range(max(256 * 256, n_wg * 1))]
    l2 = [[0, 0, 0, 0] for _ in range(256)]
    l3 = [[0, 0, 0, 0]]
    # init_idx
    for g in range(n_wg * 64):
        for i in range(4):
            idx = 4 * g + i
            if idx < size:
                idxs[0][idx] = idx
    for k in range(16):
        src_v, src_i = vals[k % 2], idxs[k % 2]
        dst_v, dst_i = vals[(k + 1) % 2], idxs[(k + 1) % 2]
        # init_off
        for wg in range(n_wg):
            wg_count = [0, 0, 0, 0]
            for lid in range(64):
                gid = 64 * wg + lid
                l_count = [0, 0, 0, 0]
                for i in range(4):
                    idx = 4 * gid + i
                    if idx < size:
                        l_count[get_val_u32(src_v[idx], k)] += 1
                for d in range(4):
                    wg_count[d] += l_count[d]
            l1[wg] = list(wg_count)
        # scan_up, level 1 (num = ceil(size/256), dispatch ceil(size/65536)) and level 2
        for level, (low, nex, num, groups) in enumerate(
                ((l1, l2, n_wg, (size + 65535) // 65536), (l2, l3, (size + 65535) // 65536, 1))):
            for wg in range(groups):
                scan_arr = []
                thread_state = []
                for lid in range(64):
                    gid = 64 * wg + lid
                    tv = [[0, 0, 0, 0] for _ in range(4)]
                    for i in range(4):
                        if 4 * gid + i < num:
                            tv[i] = list(low[4 * gid + i])
                    to = [[0, 0, 0, 0], tv[0]]
                    to.append([(a + b) & M32 for a, b in zip(to[1], tv[1])])
                    to.append([(a + b) & M32 for a, b in zip(to[2], tv[2])])
                    thread_state.append((tv, to))
                    scan_arr.append([(a + b + c + d) & M32 for a, b, c, d in zip(*tv)])
                workgroup_scan(scan_arr)
                for lid in range(64):
                    gid = 64 * wg + lid
                    tv, to = thread_state[lid]
                    for i in range(4):
                        if 4 * gid + i < len(low):
                            low[4 * gid + i] = [(a + b) & M32 for a, b in zip(scan_arr[lid], to[i])]
                    if lid == 63:
                        nex[gid // 64] = [(a + b + c) & M32 for a, b, c in zip(scan_arr[63], to[3], tv[3])]
        # scan_and_sort
        L3 = l3[0]
        for wg in range(n_wg):
            scan_arr = []
            thread_vals = []
            for lid in range(64):
                gid = 64 * wg + lid
                tv = [0, 0, 0, 0]
                for i in range(4):
                    c = 4 * gid + i
                    if c < size:
                        tv[i] = src_v[c]
                thread_vals.append(tv)
                acc = [0, 0, 0, 0]
                for i in range(4):
                    acc = [a + b for a, b in zip(acc, get_val_vec(tv[i], k))]
                scan_arr.append(acc)
            workgroup_scan(scan_arr)
            for lid in range(64):
                gid = 64 * wg + lid
                tv = thread_vals[lid]
                to = [list(scan_arr[lid])]
                for i in range(3):
                    to.append([a + b for a, b in zip(to[i], get_val_vec(tv[i], k))])
                go = [0, L3[0], L3[0] + L3[1], L3[0] + L3[1] + L3[2]]
                go = [(a + b + c) & M32 for a, b, c in zip(go, l1[gid // 64], l2[gid // (64 * 256)])]
                for i in range(4):
                    c = 4 * gid + i
                    if c < size:
                        d = get_val_u32(tv[i], k)
                        n_idx = (go[d] + to[i][d]) & M32
                        dst_i[n_idx] = src_i[c]
                        dst_v[n_idx] = tv[i]
    return np.array(vals[0], dtype=np.uint32), np.array(idxs[0], dtype=np.int32)


# ---------------------------------------------------------------- radix tree
def i32(x: int) -> int:
    x &= M32
    return x - (1 << 32) if x & 0x80000000 else x


def wgsl_div(a: int, b: int) -> int:
    if b == 0:
        return a
    if a == -(1 << 31) and b == -1:
        return a
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def dif(k1: int, k2: int) -> int:
    for i in range(32):
        mask = 1 << (31 - i)
        if (k1 & mask) != (k2 & mask):
            return i
    return -1


def radix_tree(keys: np.ndarray) -> np.ndarray:
    num = keys.size
    parents = [0] * (2 * num)
    K = [int(k) for k in keys]

    def dl(i1, i2):
        if i1 >= num or i2 >= num or i1 < 0 or i2 < 0:
            return -1
        kd = dif(K[i1], K[i2])
        if kd == -1:
            kd = 32 + dif(i1 & M32, i2 & M32)
        return kd

    for i in range(num - 1):
        x = dl(i, i + 1) - dl(i, i - 1)
        d = (x > 0) - (x < 0)
        del_min = dl(i, i - d)
        l_max = 2
        while dl(i, i + l_max * d) > del_min:
            l_max = i32(l_max * 2)
        l = 0
        t = wgsl_div(l_max, 2)
        while t > 0:
            if dl(i, i + (l + t) * d) > del_min:
                l += t
            t = wgsl_div(t, 2)
        j = i + l * d
        del_node = dl(i, j)
        s = 0
        v = 2
        t = wgsl_div(i32(l - 1 + v), v)
        while t > 0:
            if dl(i, i + (s + t) * d) > del_node:
                s += t
            v = i32(v * 2)
            t = wgsl_div(i32(l - 1 + v), v)
        gamma = i + s * d + min(d, 0)
        rx, ry = gamma, gamma + 1
        if min(i, j) == gamma:
            rx = -rx - 1
        if max(i, j) == gamma + 1:
            ry = -ry - 1
        for p in (rx, ry):
            if p >= 0:
                parents[p] = i
            else:
                parents[num + -(p + 1)] = i
    return np.array(parents, dtype=np.int32)


# ---------------------------------------------------------------- up pass
def up_pass(perm, aabb, parents, seed: int):
    """Leaf threads as state machines under a seeded random interleaving."""
    num = perm.size
    bvh = [[0] * 16 for _ in range(num)]           # 16 i32/f32-bit words per node
    f2u = lambda f: int(np.float32(f).view(np.uint32))  # noqa: E731
    u2f = lambda u: np.uint32(u).view(np.float32)       # noqa: E731
    rng = random.Random(seed)

    class T:
        pass

    threads = []
    for idx in range(num):
        t = T()
        box = aabb[perm[idx]]
        t.mn = [F(box[a]) - (F(1e-8) if F(box[a]) == 0 else F(0)) for a in range(3)]
        t.mx = [F(box[4 + a]) + (F(1e-8) if F(box[4 + a]) == 0 else F(0)) for a in range(3)]
        t.mn = [F(x) for x in t.mn]
        t.mx = [F(x) for x in t.mx]
        t.c, t.w, t.level, t.done, t.pending = idx, -(idx + 1), 0, False, None
        threads.append(t)

    live = list(range(num))
    while live:
        k = rng.randrange(len(live))
        t = threads[live[k]]
        if t.pending is not None:                  # first arrival: its stores land later
            p = t.pending
            for a in range(3):
                bvh[p][a] = f2u(t.mn[a])
                bvh[p][4 + a] = f2u(t.mx[a])
            bvh[p][3] = t.w & M32
            t.done = True
        elif not (t.w != 0 or t.level == 0):
            t.done = True
        else:
            p = int(parents[t.c + num]) if t.level == 0 else int(parents[t.c])
            sibling = bvh[p][7]
            bvh[p][7] += 1
            if sibling == 0:
                t.pending = p
            else:
                for a in range(3):
                    bvh[p][8 + a] = f2u(t.mn[a])
                    bvh[p][12 + a] = f2u(t.mx[a])
                bvh[p][11] = t.w & M32
                lmin = [u2f(bvh[p][a]) for a in range(3)]
                lmax = [u2f(bvh[p][4 + a]) for a in range(3)]
                if not (any(x == 0 for x in lmin) or any(x == 0 for x in lmax)):
                    t.mn = [wmin(t.mn[a], lmin[a]) for a in range(3)]
                    t.mx = [wmax(t.mx[a], lmax[a]) for a in range(3)]
                    t.c, t.w, t.level = p, p, t.level + 1
                # else: spin - the loop runs again from the top (:266-268)
        if t.done:
            live[k] = live[-1]
            live.pop()
    return np.array(bvh, dtype=np.uint64).astype(np.uint32)


def canonicalize(nodes: np.ndarray) -> np.ndarray:
    nodes = nodes.copy()
    n = nodes.shape[0]
    if n == 1:
        nodes[0, 15] = 0
        return nodes
    for p in range(n - 1):
        lc, rc = int(nodes[p, 3].view(np.int32)), int(nodes[p, 11].view(np.int32))
        lp = lc if lc >= 0 else -(lc + 1)
        rp = rc if rc >= 0 else -(rc + 1)
        if lp > rp:
            nodes[p, 0:8], nodes[p, 8:16] = nodes[p, 8:16].copy(), nodes[p, 0:8].copy()
        nodes[p, 7] = 2
        nodes[p, 15] = 0
    return nodes


# ---------------------------------------------------------------- traversal
def trace(nodes: np.ndarray, tris: np.ndarray, rays: np.ndarray):
    u2f = lambda u: np.uint32(u).view(np.float32)  # noqa: E731

    def sub(a, b):
        return [F(a[0] - b[0]), F(a[1] - b[1]), F(a[2] - b[2])]

    def dot(a, b):
        return F(F(F(a[0] * b[0]) + F(a[1] * b[1])) + F(a[2] * b[2]))

    def cross(a, b):
        return [F(F(a[1] * b[2]) - F(a[2] * b[1])), F(F(a[2] * b[0]) - F(a[0] * b[2])),
                F(F(a[0] * b[1]) - F(a[1] * b[0]))]

    def tri_isect(o, d, t):
        v0, v1, v2 = [F(x) for x in t[0:3]], [F(x) for x in t[4:7]], [F(x) for x in t[8:11]]
        v0v1, v0v2 = sub(v1, v0), sub(v2, v0)
        pvec = cross(d, v0v2)
        det = dot(v0v1, pvec)
        if abs(det) < F(1e-10):
            return F(-1)
        i_det = F(F(1) / det)
        tvec = sub(o, v0)
        u = F(dot(tvec, pvec) * i_det)
        if u < 0 or u > 1:
            return F(-1)
        qvec = cross(tvec, v0v1)
        v = F(dot(d, qvec) * i_det)
        if v < 0 or F(u + v) > 1:
            return F(-1)
        return F(dot(v0v2, qvec) * i_det)

    def box_isect(lo, hi, o, d):
        inv = [F(F(1) / d[a]) for a in range(3)]
        f = [F(F(hi[a] - o[a]) * inv[a]) for a in range(3)]
        nn = [F(F(lo[a] - o[a]) * inv[a]) for a in range(3)]
        tmax = [wmax(f[a], nn[a]) for a in range(3)]
        tmin = [wmin(f[a], nn[a]) for a in range(3)]
        t0 = wmax(tmin[0], wmax(tmin[1], tmin[2]))
        t1 = wmin(tmax[0], wmin(tmax[1], tmax[2]))
        if t1 >= t0:
            return F(-1e30) if t1 < 0 else t0
        return F(-1e30)

    prims, ts = [], []
    with np.errstate(all="ignore"):
        for r in rays:
            o = [F(r[0]), F(r[1]), F(r[2])]
            d = [F(r[4]), F(r[5]), F(r[6])]
            d = [F(x + (F(1e-5) if abs(x) < F(1e-5) else F(0))) for x in d]
            dist, prim = F(1e30), -1
            stack, sp, node_idx = [0] * 64, 0, 0
            while sp >= 0:
                if node_idx < 0:
                    leaf = -(node_idx + 1)
                    t = tri_isect(o, d, tris[leaf])
                    if t > 0 and t < dist:
                        dist, prim = wmin(t, dist), leaf
                    sp -= 1
                    node_idx = stack[sp] if sp >= 0 else 0
                else:
                    nd = nodes[node_idx]
                    lmin = [u2f(nd[a]) for a in range(3)]
                    lmax = [u2f(nd[4 + a]) for a in range(3)]
                    rmin = [u2f(nd[8 + a]) for a in range(3)]
                    rmax = [u2f(nd[12 + a]) for a in range(3)]
                    lc, rc = int(np.uint32(nd[3]).view(np.int32)), int(np.uint32(nd[11]).view(np.int32))
                    ld = box_isect(lmin, lmax, o, d)
                    rd = box_isect(rmin, rmax, o, d)
                    lv = ld != F(-1e30) and ld < dist
                    rv = rd != F(-1e30) and rd < dist
                    if lv and rv:
                        c, f = (lc, rc) if ld < rd else (rc, lc)
                        stack[sp] = f
                        sp += 1
                        node_idx = c
                    elif lv:
                        node_idx = lc
                    elif rv:
                        node_idx = rc
                    else:
                        sp -= 1
                        node_idx = stack[sp] if sp >= 0 else 0
            prims.append(-1 if dist == F(1e30) else prim)
            ts.append(F(-1) if dist == F(1e30) else dist)
    return np.array(prims, dtype=np.int32), np.array(ts, dtype=np.float32)


# ---------------------------------------------------------------- cases
def scene_bounds(tri):
    v = np.concatenate([tri[:, 0:3], tri[:, 4:7], tri[:, 8:11]])
    return np.concatenate([v.min(axis=0), v.max(axis=0)]).astype(np.float32)


def cases():
    out = []
    for n in (1, 2, 3, 4, 5, 7, 8, 9, 17, 63, 64, 65, 255, 256, 257, 1000):
        out.append((f"uniform_{n}", scenes.uniform_soup(n, seed=1000 + n), None))
    # all triangles identical: every key equal, the tree splits on the index tie-break
    t = scenes.uniform_soup(1, seed=7)
    out.append(("all_equal_37", np.repeat(t, 37, axis=0), None))
    # a few distinct positions repeated: long runs of duplicate keys
    base = scenes.uniform_soup(6, seed=8)
    out.append(("dup_runs_300", base[np.random.Generator(np.random.PCG64(9)).integers(0, 6, 300)], None))
    # flat scene (z = 0 everywhere): zero extent -> rel = 0/0 = NaN -> quantised 0, and
    # exactly-zero box components that the up pass nudges by 1e-8
    flat = scenes.uniform_soup(200, seed=10)
    flat[:, [2, 6, 10]] = 0.0
    out.append(("flat_z0_200", flat, None))
    # vertices exactly at the origin and on the axes
    zeros = scenes.uniform_soup(64, seed=11)
    zeros[::3, 0:3] = 0.0
    zeros[1::4, 4] = 0.0
    zeros[2::5, 9] = -0.0
    out.append(("zeros_64", zeros, None))
    # parse-obj output shape: model + two floor triangles far outside the host bounds
    tri, b = scenes.obj_like_with_floor(510, seed=12)
    out.append(("obj_floor_512", tri, b))
    # host bounds narrower than the scene on one axis (keys above 2^30)
    tri = scenes.uniform_soup(128, seed=13)
    out.append(("narrow_bounds_128", tri, np.array([0.25, 0.0, 0.0, 0.75, 1.0, 1.0], np.float32)))
    # the displaced sphere at 32 x 32 quads
    out.append(("sphere_2048", scenes.sphere_mesh(32, seed=14), None))
    out.append(("uniform_4096", scenes.uniform_soup(4096, seed=15), None))
    return out


def make_rays(n, seed, radius=3.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    o = rng.standard_normal((n, 3))
    o = o / np.linalg.norm(o, axis=1, keepdims=True) * radius
    tgt = rng.uniform(-1.0, 1.0, (n, 3))
    d = tgt - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), dtype=np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    return rays


def main():
    data = {}
    names = []
    for ci, (name, tri, bounds) in enumerate(cases()):
        tri = np.ascontiguousarray(tri, dtype=np.float32)
        b = scene_bounds(tri) if bounds is None else bounds
        aabb, keys = aabb_z_idx(tri, b)
        skeys, perm = radix_sort(keys)
        parents = radix_tree(skeys)
        nodes = canonicalize(up_pass(perm, aabb, parents, seed=ci))
        otri = tri[perm]
        names.append(name)
        data[f"{name}/tri"] = tri
        data[f"{name}/host_bounds"] = (bounds if bounds is not None else np.zeros(0, np.float32))
        data[f"{name}/bounds"] = b
        data[f"{name}/keys_unsorted"] = keys
        data[f"{name}/morton"] = skeys
        data[f"{name}/leaf_index"] = perm.view(np.uint32)
        data[f"{name}/parents"] = parents
        data[f"{name}/nodes"] = nodes
        data[f"{name}/tris"] = otri
        if name in ("uniform_1000", "sphere_2048", "obj_floor_512"):
            rays = make_rays(256, seed=ci)
            if name == "sphere_2048":
                rays[:, 0:3] *= 1.0
            prim, t = trace(nodes, otri, rays)
            data[f"{name}/rays"] = rays
            data[f"{name}/hit_prim"] = prim
            data[f"{name}/hit_t"] = t
        print(name, tri.shape[0], "ok", flush=True)
    # hand-derived Morton known answers (aabb-z-idx.js:197-209)
    kat_in = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1023, 0, 0], [1023, 1023, 1023],
                       [512, 256, 128], [1024, 0, 0], [0xFFFFFFFF, 0, 0]], dtype=np.uint32)
    data["kat/morton_in"] = kat_in
    data["kat/morton_out"] = np.array([morton_code(*map(int, r)) for r in kat_in], dtype=np.uint32)
    data["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **data)


if __name__ == "__main__":
    main()
