"""Parity of the sm_100a build (through the C ABI) with the oracle and the golden fixtures.

Bit-exact everywhere: Morton keys, permutation, parent links, every word of every BVHNode
(canonical slot order) and every word of the rearranged triangles.  Traversal parity compares
hit primitive and the bits of t.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("morton", "leaf_index", "parents", "nodes", "tris")


def as_u32(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype.itemsize == 4 else a


def assert_same(got: dict, ref: dict, tag=""):
    for f in FIELDS:
        g, r = as_u32(got[f]).reshape(-1), as_u32(ref[f]).reshape(-1)
        assert g.shape == r.shape, f"{tag} {f}: shape {g.shape} vs {r.shape}"
        bad = np.nonzero(g != r)[0]
        assert bad.size == 0, f"{tag} {f}: {bad.size} words differ, first at {bad[:8]}"


def build_np(builder, tri, bounds=None, host=False, **kw):
    import torch
    if host:
        res = builder.build_soup(tri, bounds, **kw)
    else:
        res = builder.build_soup(torch.from_numpy(np.ascontiguousarray(tri)).cuda(), bounds, **kw)
    return res, res.to_numpy()


def golden_case(golden, name):
    ref = {f: golden[f"{name}/{f}"] for f in FIELDS}
    hb = golden[f"{name}/host_bounds"]
    return golden[f"{name}/tri"], (hb if hb.size else None), ref


def test_library_is_in_tree():
    import os
    import lvbh
    assert os.path.dirname(lvbh._native.LIB_PATH).endswith(os.path.join("webgpu-lvbh-demo_b200", "lvbh"))
    assert "sm_100a" in lvbh.version()


@pytest.mark.parametrize("host", [False, True])
def test_golden_cases(builder, golden, host):
    for name in golden["names"]:
        tri, hb, ref = golden_case(golden, name)
        _, got = build_np(builder, tri, hb, host=host)
        assert_same(got, ref, name)
        np.testing.assert_array_equal(got["bounds"].view(np.uint32), golden[f"{name}/bounds"].view(np.uint32))


def test_golden_traces(builder, golden):
    import torch
    for name in golden["names"]:
        if f"{name}/rays" not in golden:
            continue
        tri, hb, _ = golden_case(golden, name)
        res, _ = build_np(builder, tri, hb)
        prim, t, st = builder.trace(res, torch.from_numpy(golden[f"{name}/rays"]).cuda())
        np.testing.assert_array_equal(prim.cpu().numpy(), golden[f"{name}/hit_prim"])
        np.testing.assert_array_equal(t.cpu().numpy().view(np.uint32), golden[f"{name}/hit_t"].view(np.uint32))


@pytest.mark.parametrize("n", [0, 1, 2, 3, 31, 32, 33, 511, 512, 513, 1025, 4095, 4096, 4097, 8191, 8193,
                               12289, 65535, 65537, 100_003, 262_145])
def test_sizes_vs_oracle(builder, n):
    import oracle
    from lvbh import scenes
    tri = scenes.uniform_soup(n, seed=n + 17)
    _, got = build_np(builder, tri)
    ref = oracle.build(tri, None, threads=0)
    assert_same(got, ref, f"n={n}")
    if n:
        np.testing.assert_array_equal(got["bounds"].view(np.uint32), ref["bounds"].view(np.uint32))


def test_uniform_65536_soup_and_indexed(builder):
    """The 65,536-triangle uniform workload, as a soup and as an indexed mesh."""
    import oracle
    from lvbh import scenes
    tri = scenes.uniform_soup(65_536, seed=0)
    ref = oracle.build(tri, None, threads=0)
    _, got = build_np(builder, tri)
    assert_same(got, ref, "soup")
    xyz, idx3 = scenes.indexed_from_soup(tri)
    ref_i = oracle.build(oracle.gather_indexed(xyz, idx3), None, threads=0)
    got_h = builder.build_indexed(xyz, idx3).to_numpy()
    assert_same(got_h, ref_i, "indexed host")
    import torch
    got_d = builder.build_indexed(torch.from_numpy(xyz).cuda(), torch.from_numpy(idx3.view(np.int32)).cuda()).to_numpy()
    assert_same(got_d, ref_i, "indexed device")
    # pads differ (3.1415 vs 0) but nothing else
    for f in ("morton", "leaf_index", "parents", "nodes"):
        np.testing.assert_array_equal(as_u32(got[f]), as_u32(got_h[f]))


def test_all_equal_keys_large(builder):
    import oracle
    from lvbh import scenes
    tri = np.repeat(scenes.uniform_soup(1, seed=3), 100_000, axis=0)
    _, got = build_np(builder, tri)
    assert_same(got, oracle.build(tri, None, threads=0), "all-equal")


def test_host_bounds_with_floor(builder):
    """parse-obj output: the floor triangles reach far outside the host bounds; with the z
    range of the bounds narrowed as well, quantised coordinates run past 1023 and alias
    through split_3's masks (keys still stay below 2^30: the last mask tops out at bit 27)."""
    import oracle
    from lvbh import scenes
    tri, b = scenes.obj_like_with_floor(200_000, seed=21)
    for bounds in (b, np.array([b[0], b[1], b[2], b[3], b[4], np.float32(0.25)], np.float32)):
        _, got = build_np(builder, tri, bounds)
        ref = oracle.build(tri, bounds, threads=0)
        assert (ref["morton"] < (1 << 30)).all()
        assert_same(got, ref, "floor")


def test_nonfinite_rejected(builder):
    import lvbh
    from lvbh import scenes
    tri = scenes.uniform_soup(5000, seed=4)
    tri[1234, 5] = np.nan
    with pytest.raises(lvbh.LvbhError) as e:
        build_np(builder, tri)
    assert e.value.code == lvbh._native.EINVAL
    tri[1234, 5] = np.inf
    with pytest.raises(lvbh.LvbhError):
        build_np(builder, tri)
    # the context stays usable
    tri[1234, 5] = 0.5
    build_np(builder, tri)


def test_failed_async_build_status_reaches_next_build():
    """A failing LVBH_ASYNC build (non-finite vertex) followed by a second build without
    lvbh_sync: the second call returns the first one's status and starts nothing; the call
    after that builds normally."""
    import ctypes

    import torch
    import lvbh
    import oracle
    from lvbh import _native, scenes
    L = _native.lib
    b = lvbh.BVHBuilder(0)
    try:
        bad = scenes.uniform_soup(5000, seed=4)
        bad[77, 9] = np.nan
        good = scenes.uniform_soup(7000, seed=5)
        keep = []

        def call(tri, flags):
            t = torch.from_numpy(tri).cuda()
            outs = lvbh.empty_outputs(tri.shape[0], t.device)
            r = lvbh._result_struct(outs, tri.shape[0])
            keep.append((t, outs, r))
            return L.lvbh_build_soup(b.ctx, ctypes.c_void_p(t.data_ptr()), tri.shape[0], None,
                                     _native.OUT_CALLER | flags, ctypes.byref(r), None), outs

        rc, _ = call(bad, _native.ASYNC)
        assert rc == _native.OK
        rc, _ = call(good, 0)
        assert rc == _native.EINVAL
        assert b"earlier LVBH_ASYNC build failed" in L.lvbh_last_error(b.ctx)
        assert L.lvbh_sync(b.ctx) == _native.OK  # nothing pending any more
        rc, outs = call(good, 0)
        assert rc == _native.OK
        assert_same({k: v.cpu().numpy() for k, v in outs.items()}, oracle.build(good, None, threads=0), "after")
    finally:
        b.close()


def test_indexed_bad_index_rejected(builder):
    import torch
    import lvbh
    from lvbh import scenes
    xyz, idx3 = scenes.indexed_from_soup(scenes.uniform_soup(1000, seed=5))
    idx3 = idx3.copy()
    idx3[10, 1] = xyz.shape[0] + 7
    with pytest.raises(lvbh.LvbhError):
        builder.build_indexed(xyz, idx3)
    with pytest.raises(lvbh.LvbhError):
        builder.build_indexed(torch.from_numpy(xyz).cuda(), torch.from_numpy(idx3.view(np.int32)).cuda())


def test_graph_replay_async_and_reuse(builder):
    """Same shape twice (graph replay), async + sync, then a larger build on the same context."""
    import torch
    import oracle
    from lvbh import scenes, empty_outputs
    tri = scenes.uniform_soup(30_000, seed=6)
    ref = oracle.build(tri, None, threads=0)
    dtri = torch.from_numpy(tri).cuda()
    outs = empty_outputs(30_000, builder.device)
    for _ in range(3):
        builder.build_soup(dtri, None, outputs=outs, sync=False)
        builder.sync()
        assert_same({k: v.cpu().numpy() for k, v in outs.items()}, ref, "replay")
    res = builder.build_soup(dtri, None, graph=False, profile=True)
    assert set(res.stage_ms) == {"upload", "bounds", "morton", "sort", "gather", "tree", "top"}
    assert_same(res.to_numpy(), ref, "profiled")
    big = scenes.uniform_soup(300_000, seed=7)
    _, got = build_np(builder, big)
    assert_same(got, oracle.build(big, None, threads=0), "grown arena")


def test_reference_shaped_entry(builder):
    """initBVHBuild(device).build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS) with a list input."""
    import lvbh
    import oracle
    from lvbh import scenes
    tri, b = scenes.obj_like_with_floor(2000, seed=8)
    bounds = {"min": [float(x) for x in b[:3]], "max": [float(x) for x in b[3:]]}
    out = builder.build(tri.ravel().tolist(), tri.shape[0], bounds)
    ref = oracle.build(tri, b, threads=0)
    np.testing.assert_array_equal(out["BVH_BUFFER"].cpu().numpy().view(np.uint32), ref["nodes"])
    np.testing.assert_array_equal(out["O_TRIANGLE_BUFFER"].cpu().numpy().view(np.uint32), ref["tris"].view(np.uint32))
    with pytest.raises(ValueError):
        builder.build(tri.ravel().tolist() + [1.0], tri.shape[0], bounds)
    short = builder.build(tri.ravel()[:-12].tolist(), tri.shape[0], bounds)   # last triangle zero
    t2 = tri.copy()
    t2[-1] = 0
    np.testing.assert_array_equal(short["BVH_BUFFER"].cpu().numpy().view(np.uint32), oracle.build(t2, b)["nodes"])
    assert isinstance(lvbh.initBVHBuild(0), lvbh.BVHBuilder)


def test_sphere_2M_and_1M_rays(builder):
    """2,097,152-triangle displaced sphere: bit-exact build, then 1M rays traced through both
    trees return identical hits (CUDA traversal over the CUDA tree vs the oracle's traversal
    over the oracle tree)."""
    import torch
    import oracle
    from lvbh import scenes
    tri = scenes.sphere_mesh(1024, seed=1)
    ref = oracle.build(tri, None, threads=0)
    dup = 1.0 - np.unique(ref["morton"]).size / ref["morton"].size
    res, got = build_np(builder, tri)
    assert_same(got, ref, "sphere")
    rays = make_rays(1 << 20, seed=11)
    prim, t, st = builder.trace(res, torch.from_numpy(rays).cuda())
    rp, rt, rs = oracle.trace(ref["nodes"], ref["tris"], rays, threads=0)
    np.testing.assert_array_equal(prim.cpu().numpy(), rp)
    np.testing.assert_array_equal(t.cpu().numpy().view(np.uint32), rt.view(np.uint32))
    np.testing.assert_array_equal(st.cpu().numpy().view(np.uint32), rs)
    hits = int((rp >= 0).sum())
    print(f"sphere: duplicate-key fraction {dup:.3f}, hits {hits}/{rays.shape[0]}, "
          f"max stack {int(rs.max())} (reference stack: 32)")
    assert hits > rays.shape[0] // 4


def test_clustered_16M(builder):
    """2^24-triangle Gaussian-mixture scene, bit-exact against the oracle, plus the
    size-independent tree properties."""
    from lvbh import scenes
    import oracle
    tri = scenes.clustered_soup(1 << 24, seed=2)
    res, got = build_np(builder, tri)
    ref = oracle.build(tri, None, threads=0)
    assert_same(got, ref, "clustered")
    check_tree_properties(tri, got)


def make_rays(n, seed, radius=3.0):
    from lvbh import scenes
    return scenes.sphere_rays(n, seed, radius)


def check_tree_properties(tri, got):
    """Sorted keys, stable bijective permutation, one parent per node, two children per
    internal node, node boxes = exact min/max of their children, leaf boxes = triangle boxes."""
    n = tri.shape[0]
    keys, perm = got["morton"], got["leaf_index"].astype(np.int64)
    assert (keys[1:] >= keys[:-1]).all()
    assert np.bincount(perm, minlength=n).max() == 1
    eq = keys[1:] == keys[:-1]
    assert (perm[1:][eq] > perm[:-1][eq]).all()          # stability
    nodes = got["nodes"][: n - 1]
    lc = nodes[:, 3].view(np.int32).astype(np.int64)
    rc = nodes[:, 11].view(np.int32).astype(np.int64)
    ch = np.concatenate([lc, rc])
    leaf = ch < 0
    assert np.bincount(-(ch[leaf] + 1), minlength=n).max() == 1 and leaf.sum() == n
    assert np.bincount(ch[~leaf], minlength=n - 1)[1:].max() == 1 and (~leaf).sum() == n - 2
    par = got["parents"]
    idx = np.arange(n - 1)
    assert (par[n + (-(lc[lc < 0] + 1))] == idx[lc < 0]).all()
    assert (par[lc[lc >= 0]] == idx[lc >= 0]).all()
    f = got["nodes"].view(np.float32)
    # internal children: the child's merged box equals the slot box in the parent
    for side, c in ((0, lc), (8, rc)):
        m = c >= 0
        kids = f[c[m]]
        box_min = np.minimum(kids[:, 0:3], kids[:, 8:11])
        box_max = np.maximum(kids[:, 4:7], kids[:, 12:15])
        np.testing.assert_array_equal(f[idx[m], side:side + 3], box_min)
        np.testing.assert_array_equal(f[idx[m], side + 4:side + 7], box_max)
        lm = ~m
        t = tri[perm[-(c[lm] + 1)]]
        bmin = np.minimum(t[:, 0:3], np.minimum(t[:, 4:7], t[:, 8:11]))
        bmax = np.maximum(t[:, 0:3], np.maximum(t[:, 4:7], t[:, 8:11]))
        bmin = np.where(bmin == 0, np.float32(-1e-8), bmin)
        bmax = np.where(bmax == 0, np.float32(1e-8), bmax)
        np.testing.assert_array_equal(f[idx[lm], side:side + 3], bmin)
        np.testing.assert_array_equal(f[idx[lm], side + 4:side + 7], bmax)


def test_shrinking_builds_on_one_context(builder):
    """Builds of shrinking sizes on one context: scratch laid out for an earlier, larger build
    (open-item lists, level counters of the straddling pass) must not leak into a later one."""
    from lvbh import scenes
    for n in (1 << 20, 300_001, 131_072, 70_001, 5000):
        tri = scenes.clustered_soup(n, seed=n % 97)
        _, got = build_np(builder, tri)
        assert_same(got, oracle_build(tri), f"n={n}")


def oracle_build(tri):
    import oracle
    return oracle.build(tri, None, threads=0)


def test_chunked_host_upload(builder):
    """A host soup of 2^21 + 4099 triangles is uploaded in chunks, each chunk's first pass (the
    box and centroids, or with host bounds the Morton keys) running while the next chunk is
    copied: bit-exact against the oracle and the device-input build, from pageable and pinned
    host memory, after an LVBH_ASYNC build that still reads the staging buffer, again on graph
    replay, and with MODEL_BOUNDS wider than the scene."""
    import torch
    from lvbh import scenes
    import oracle
    n = (1 << 21) + 4099
    tri = scenes.clustered_soup(n, seed=12)
    ref = oracle.build(tri, None, threads=0)
    _, dev = build_np(builder, tri)
    assert_same(dev, ref, "device input")
    other = scenes.clustered_soup(n, seed=13)
    pending = builder.build_soup(other, None, sync=False)
    _, got = build_np(builder, tri, host=True)
    assert_same(got, ref, "chunked upload after an async build")
    del pending
    pinned = torch.from_numpy(tri).pin_memory()
    for tag in ("pinned", "pinned, replayed"):
        _, got = build_np(builder, pinned.numpy(), host=True)
        assert_same(got, ref, tag)
    # with MODEL_BOUNDS the Morton keys of each chunk are made while the next chunk is copied
    hb = oracle.scene_bounds(tri)
    hb[:3] -= np.float32(0.25)
    hb[3:] += np.float32(0.5)
    ref_hb = oracle.build(tri, hb, threads=0)
    _, got = build_np(builder, pinned.numpy(), hb, host=True)
    assert_same(got, ref_hb, "chunked upload with host bounds")
    _, got = build_np(builder, tri, hb)
    assert_same(got, ref_hb, "device input with host bounds")


def test_caller_outputs_one_element_off_16_bytes(builder):
    """Caller-provided result buffers need 16-byte alignment only for nodes and tris; parents,
    leaf_index and morton may start anywhere 4-byte aligned, as slices of a larger buffer do
    when meshes are built one by one into it.  With those three one element past a 16-byte
    boundary (and in the sort's ping-pong, where leaf_index is read back as the values of the
    second pass) the build stays bit-exact."""
    import torch
    import oracle
    from lvbh import scenes
    n = 70_001
    tri = scenes.clustered_soup(n, seed=31)
    dev = torch.device("cuda")
    outs = {"nodes": torch.empty((n, 16), dtype=torch.int32, device=dev),
            "tris": torch.empty((n, 12), dtype=torch.float32, device=dev),
            "parents": torch.empty(2 * n + 1, dtype=torch.int32, device=dev)[1:],
            "leaf_index": torch.empty(n + 1, dtype=torch.int32, device=dev)[1:],
            "morton": torch.empty(n + 3, dtype=torch.int32, device=dev)[3:]}
    for k in ("parents", "leaf_index", "morton"):
        assert outs[k].data_ptr() % 16 != 0
    builder.build_soup(torch.from_numpy(tri).cuda(), None, outputs=outs)
    got = {k: v.cpu().numpy() for k, v in outs.items()}
    assert_same(got, oracle.build(tri, None, threads=0), "outputs off 16-byte boundaries")
