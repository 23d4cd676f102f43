"""Nodes that straddle tree blocks, in numbers the group level of the straddling pass cannot hold.

The tree pass builds each block of 256 sorted leaves on its own; what leaves a block (a complete
subtree whose parent crosses the block's edge) is an open item, and the straddling pass climbs
the open items of 16 consecutive blocks in shared memory when they number at most 256, else
hands all of them to the global pass unchanged.  Uniform or clustered scenes leave about 8 items
per block, so that second branch only runs on scenes like this one: around every block
boundary the Morton keys zig-zag - the common prefix of neighbouring keys shrinks by one bit per
step, alternately to the left and to the right of the boundary - so every node on the path above
the boundary crosses it and each side leaves about ten items.  The CPU test checks that premise
from the keys alone (Karras tree of the sorted keys, index tie-break); the GPU test checks the
build bit-exact against the oracle.
"""
import numpy as np
import pytest

EB = 256           # leaves per tree block
GROUP_BLOCKS = 16  # blocks per group of the straddling pass
GROUP_CAP = 256    # open items one group climbs in shared memory
LOW = 20           # zig-zag bits below the group's high part


def zigzag_low_keys():
    """(left part, right part) of one zig-zag in the low LOW bits, each in ascending order;
    the boundary falls between them."""
    c = sum(1 << b for b in range(1, LOW, 2)) | 1
    left, lo = [c - 1], c - 1
    for b in range(1, LOW, 2):  # clear bit b (set in lo) and everything below it
        assert lo >> b & 1
        lo &= ~((2 << b) - 1)
        left.append(lo)
    right, hi = [c], c
    for b in range(2, LOW - 1, 2):  # set bit b (clear in hi), clear everything below it
        assert not hi >> b & 1
        hi = (hi | (1 << b)) & ~((1 << b) - 1)
        right.append(hi)
    return sorted(left), right


def zigzag_keys(blocks=512):
    """Sorted 30-bit keys: block j holds the right part of zig-zag j, filler, and the left part
    of zig-zag j + 1, so that every inner block boundary is a zig-zag centre."""
    left, right = zigzag_low_keys()
    keys = []
    for j in range(blocks):
        part = []
        if j > 0:
            part += [((2 * j - 1) << LOW) | v for v in right]
        nfill = EB - len(part) - (len(left) if j < blocks - 1 else 0)
        fill = np.linspace(0, (1 << LOW) - 1, nfill).astype(np.int64)
        part += [((2 * j) << LOW) | int(v) for v in fill]
        if j < blocks - 1:
            part += [((2 * j + 1) << LOW) | v for v in left]
        assert len(part) == EB
        keys += part
    k = np.array(keys, dtype=np.int64)
    assert np.all(np.diff(k) > 0) and k.max() < (1 << 30)
    return k.astype(np.uint32)


def soup_from_keys(keys, seed=5):
    """One degenerate triangle per key at the centre of its Morton cell (bounds [0, 1]^3), in a
    seeded random input order."""
    k = keys.astype(np.uint32)
    q = np.zeros((k.size, 3), np.uint32)
    for bit in range(10):
        for a in range(3):
            q[:, a] |= ((k >> np.uint32(3 * bit + a)) & np.uint32(1)) << np.uint32(bit)
    c = ((q.astype(np.float64) + 0.5) / 1024.0).astype(np.float32)  # exact binary fractions
    tri = np.zeros((k.size, 12), np.float32)
    for v in range(3):
        tri[:, 4 * v:4 * v + 3] = c
    order = np.random.default_rng(seed).permutation(k.size)
    return tri[order], np.array([0, 0, 0, 1, 1, 1], np.float32)


def open_items_per_block(keys):
    """Open items each block leaves: complete children (range inside one block) of nodes whose
    range crosses a block edge, in the Karras tree of the sorted keys (index tie-break)."""
    k = keys.astype(np.int64)
    n = k.size
    x = k[:-1] ^ k[1:]
    d = np.where(x != 0, 32 - np.floor(np.log2(np.maximum(x, 1))).astype(np.int64) - 1, 0)
    same = x == 0
    if same.any():
        g = np.arange(n - 1, dtype=np.int64)
        gx = g ^ (g + 1)
        d[same] = 32 + 32 - np.floor(np.log2(gx[same])).astype(np.int64) - 1
    d = list(d)
    left = [-1] * (n - 1)  # nearest split to the left with a smaller d (-1 past the start)
    stack = []
    for s in range(n - 1):
        while stack and d[stack[-1]] > d[s]:
            stack.pop()
        left[s] = stack[-1] if stack else -1
        stack.append(s)
    right = [n - 1] * (n - 1)  # nearest split to the right with a smaller d (n - 1 past the end)
    stack = []
    for s in range(n - 2, -1, -1):
        while stack and d[stack[-1]] > d[s]:
            stack.pop()
        right[s] = stack[-1] if stack else n - 1
        stack.append(s)
    items = np.zeros((n + EB - 1) // EB, np.int64)
    for s in range(n - 1):
        lo, hi = left[s] + 1, right[s]
        if lo // EB == hi // EB:
            continue
        for a, b in ((lo, s), (s + 1, hi)):
            if a // EB == b // EB:
                items[a // EB] += 1
    return items


def test_zigzag_premise():
    """CPU: the scene makes groups of 16 blocks with more open items than one group climbs."""
    keys = zigzag_keys()
    items = open_items_per_block(keys)
    groups = np.add.reduceat(items, np.arange(0, items.size, GROUP_BLOCKS))
    assert items[1:-1].min() >= 16, items[:8]
    assert groups.max() > GROUP_CAP, groups
    # and the triangles quantise to exactly these keys
    import oracle
    tri, bounds = soup_from_keys(keys[:4096])
    got = oracle.build(tri, bounds, threads=0)["morton"]
    np.testing.assert_array_equal(np.asarray(got, np.uint32), keys[:4096])


@pytest.mark.gpu
def test_zigzag_build_vs_oracle(builder):
    """GPU: the build of the zig-zag scene (131,072 triangles, every group past the cap) is
    bit-exact against the oracle."""
    import oracle
    from test_parity_gpu import assert_same, build_np
    keys = zigzag_keys()
    tri, bounds = soup_from_keys(keys)
    ref = oracle.build(tri, bounds, threads=0)
    np.testing.assert_array_equal(np.asarray(ref["morton"], np.uint32), keys)
    _, got = build_np(builder, tri, bounds)
    assert_same(got, ref, "zig-zag")
    _, got_h = build_np(builder, tri, bounds, host=True)
    assert_same(got_h, ref, "zig-zag host")
