"""The oracle pinned against the golden fixtures (a literal simulation of the reference WGSL),
hand-derived known answers, and independent restatements of each step.  CPU only."""
import numpy as np
import pytest

import oracle
from lvbh import scenes


def test_oracle_matches_golden(golden):
    for name in golden["names"]:
        tri = golden[f"{name}/tri"]
        hb = golden[f"{name}/host_bounds"]
        o = oracle.build(tri, hb if hb.size else None, threads=1)
        for f in ("morton", "leaf_index", "parents", "nodes", "tris"):
            np.testing.assert_array_equal(np.ascontiguousarray(o[f]).view(np.uint32),
                                          np.ascontiguousarray(golden[f"{name}/{f}"]).view(np.uint32),
                                          err_msg=f"{name}/{f}")
        np.testing.assert_array_equal(o["bounds"], golden[f"{name}/bounds"])
        aabb, keys = oracle.aabb_zidx(tri, golden[f"{name}/bounds"])
        np.testing.assert_array_equal(keys, golden[f"{name}/keys_unsorted"])


def test_oracle_traces_match_golden(golden):
    checked = 0
    for name in golden["names"]:
        if f"{name}/rays" not in golden:
            continue
        p, t, _ = oracle.trace(golden[f"{name}/nodes"], golden[f"{name}/tris"], golden[f"{name}/rays"])
        np.testing.assert_array_equal(p, golden[f"{name}/hit_prim"])
        np.testing.assert_array_equal(t.view(np.uint32), golden[f"{name}/hit_t"].view(np.uint32))
        checked += int((p >= 0).sum())
    assert checked > 100


def test_morton_known_answers(golden):
    # split_3(1023) = 0x09249249; all axes at 1023 -> 0x3FFFFFFF; z is the most significant
    kin, kout = golden["kat/morton_in"], golden["kat/morton_out"]
    hand = {(0, 0, 0): 0, (1, 0, 0): 1, (0, 1, 0): 2, (0, 0, 1): 4, (1023, 0, 0): 0x09249249,
            (1023, 1023, 1023): 0x3FFFFFFF}
    for row, out in zip(kin, kout):
        key = tuple(int(x) for x in row)
        if key in hand:
            assert int(out) == hand[key], key
    # a centroid exactly at the max corner quantises to 1023 on every axis
    tri = np.zeros((2, 12), np.float32)
    tri[1, [0, 1, 2, 4, 5, 6, 8, 9, 10]] = 1.0
    _, keys = oracle.aabb_zidx(tri, np.array([0, 0, 0, 1, 1, 1], np.float32))
    assert list(keys) == [0, 0x3FFFFFFF]


@pytest.mark.parametrize("n,bits", [(1, 30), (1000, 30), (70_000, 32), (200_003, 8)])
def test_sort_is_stable_argsort(n, bits):
    rng = np.random.Generator(np.random.PCG64(n))
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    sk, perm = oracle.radix_sort(keys)
    ref = np.argsort(keys, kind="stable")
    np.testing.assert_array_equal(perm, ref)
    np.testing.assert_array_equal(sk, keys[ref])


def test_threaded_oracle_equals_sequential():
    tri = scenes.clustered_soup(300_000, seed=9)
    a = oracle.build(tri, None, threads=1)
    b = oracle.build(tri, None, threads=0)
    for k in a:
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)


def _karras_reference(keys):
    """Textbook Karras (2012) over (key, index), written independently of the WGSL loop."""
    n = keys.size

    def dl(i, j):
        if j < 0 or j >= n:
            return -1
        a, b = int(keys[i]), int(keys[j])
        return (32 - (a ^ b).bit_length()) if a != b else 32 + (32 - (i ^ j).bit_length())

    parents = np.zeros(2 * n, np.int32)
    for i in range(n - 1):
        d = 1 if dl(i, i + 1) - dl(i, i - 1) > 0 else -1
        dmin = dl(i, i - d)
        lmax = 2
        while dl(i, i + lmax * d) > dmin:
            lmax *= 2
        l, t = 0, lmax // 2
        while t >= 1:
            if dl(i, i + (l + t) * d) > dmin:
                l += t
            t //= 2
        j = i + l * d
        dn = dl(i, j)
        s, div = 0, 2
        while True:
            t = -(-l // div)
            if dl(i, i + (s + t) * d) > dn:
                s += t
            if t <= 1:
                break
            div *= 2
        g = i + s * d + min(d, 0)
        parents[n + g if min(i, j) == g else g] = i
        parents[n + g + 1 if max(i, j) == g + 1 else g + 1] = i
    return parents


@pytest.mark.parametrize("n,spread", [(2, 10), (50, 4), (300, 1 << 30), (777, 16)])
def test_radix_tree_equals_textbook_karras(n, spread):
    rng = np.random.Generator(np.random.PCG64(n))
    keys = np.sort(rng.integers(0, spread, n).astype(np.uint32))
    np.testing.assert_array_equal(oracle.radix_tree(keys), _karras_reference(keys))


def test_up_pass_boxes_equal_subtree_minmax():
    """Canonical node boxes = exact min/max over the leaves of each subtree (nudged)."""
    tri = scenes.uniform_soup(3000, seed=12)
    o = oracle.build(tri, None)
    n = tri.shape[0]
    nodes = o["nodes"]
    f = nodes.view(np.float32)
    t = tri[o["leaf_index"].astype(np.int64)]
    lmin = np.minimum(t[:, 0:3], np.minimum(t[:, 4:7], t[:, 8:11]))
    lmax = np.maximum(t[:, 0:3], np.maximum(t[:, 4:7], t[:, 8:11]))
    lmin = np.where(lmin == 0, np.float32(-1e-8), lmin)
    lmax = np.where(lmax == 0, np.float32(1e-8), lmax)

    def box(c):
        if c < 0:
            k = -(c + 1)
            return lmin[k], lmax[k], k, k
        a0, a1, al, ar = box(int(nodes[c, 3].view(np.int32)))
        b0, b1, bl, br = box(int(nodes[c, 11].view(np.int32)))
        assert ar + 1 == bl                         # left slot covers the lower range
        np.testing.assert_array_equal(f[c, 0:3], a0)
        np.testing.assert_array_equal(f[c, 4:7], a1)
        np.testing.assert_array_equal(f[c, 8:11], b0)
        np.testing.assert_array_equal(f[c, 12:15], b1)
        assert nodes[c, 7] == 2 and nodes[c, 15] == 0
        return np.minimum(a0, b0), np.maximum(a1, b1), al, br

    import sys
    sys.setrecursionlimit(10000)
    _, _, lo, hi = box(0)
    assert (lo, hi) == (0, n - 1)
    assert (nodes[n - 1] == 0).all()


def test_rearrange_and_indexed_gather():
    tri = scenes.uniform_soup(500, seed=13)
    perm = np.random.Generator(np.random.PCG64(1)).permutation(500).astype(np.int32)
    np.testing.assert_array_equal(oracle.rearrange(tri, perm), tri[perm])
    xyz, idx3 = scenes.indexed_from_soup(tri)
    g = oracle.gather_indexed(xyz, idx3)
    t2 = tri.copy()
    t2[:, [3, 7, 11]] = 0
    np.testing.assert_array_equal(g, t2)


def test_empty_and_single():
    o = oracle.build(np.zeros((0, 12), np.float32))
    assert o["nodes"].shape == (0, 16)
    tri = scenes.uniform_soup(1, seed=2)
    o = oracle.build(tri)
    assert o["nodes"][0, 3].view(np.int32) == -1 and o["nodes"][0, 7] == 1
    assert (o["nodes"][0, 8:] == 0).all() and (o["parents"] == 0).all()
