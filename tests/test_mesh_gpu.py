"""The indexed leaf format (lvbh_build_mesh / lvbh_trace_mesh, through the C ABI).

The tree of an indexed mesh built without any 48-byte triangle copy must equal, word for word,
the soup build of the triangles the mesh spells out (and so the oracle's): Morton keys,
permutation, parent links, every BVHNode word and the quantisation box; the leaf rows must be
the index triples of the sorted triangles; traversal through the indexed leaves must return the
same hit primitives and t bits as traversal through the sorted soup.
"""
import numpy as np
import pytest

import oracle
from test_parity_gpu import as_u32

pytestmark = pytest.mark.gpu

TREE = ("morton", "leaf_index", "parents", "nodes")


def mesh_of(quads, seed, extra_far_vertices=0):
    from lvbh import scenes
    xyz, idx = scenes.sphere_mesh(quads, seed=seed, indexed=True)
    v4 = np.zeros((xyz.shape[0] + extra_far_vertices, 4), np.float32)
    v4[: xyz.shape[0], :3] = xyz
    v4[xyz.shape[0]:, :3] = 1000.0  # rows no triangle uses: they must not widen the box
    return v4, idx.astype(np.uint32)


def soup_of(v4, idx):
    tri = np.zeros((idx.shape[0], 12), np.float32)
    for k in range(3):
        tri[:, 4 * k:4 * k + 3] = v4[idx[:, k], :3]
    return tri


def check_same_tree(got, ref, tag):
    for f in TREE:
        g, r = as_u32(got[f]).reshape(-1), as_u32(ref[f]).reshape(-1)
        assert g.shape == r.shape and np.array_equal(g, r), f"{tag} {f}"
    np.testing.assert_array_equal(got["bounds"].view(np.uint32), ref["bounds"].view(np.uint32))


@pytest.mark.parametrize("host", [False, True])
def test_mesh_equals_soup_build(builder, host):
    import torch
    v4, idx = mesh_of(128, 3, extra_far_vertices=17)
    if host:
        res = builder.build_mesh(v4, idx)
    else:
        res = builder.build_mesh(torch.from_numpy(v4).cuda(), torch.from_numpy(idx.view(np.int32)).cuda())
    got = res.to_numpy()
    tri = soup_of(v4, idx)
    ref = builder.build_soup(torch.from_numpy(tri).cuda()).to_numpy()
    check_same_tree(got, ref, "mesh vs soup")
    np.testing.assert_array_equal(got["tris"].view(np.uint32), idx[got["leaf_index"]])
    orc = oracle.build(tri, None, threads=0)
    check_same_tree(got, orc, "mesh vs oracle")


def test_given_bounds_sizes_and_replay(builder):
    import torch
    for quads, seed in ((1, 1), (2, 2), (11, 3), (48, 4), (48, 5)):  # 2 .. 4608 triangles; replayed graph
        v4, idx = mesh_of(quads, seed)
        b = np.array([-1.5, -1.5, -1.5, 1.5, 1.5, 1.5], np.float32)
        got = builder.build_mesh(torch.from_numpy(v4).cuda(), torch.from_numpy(idx.view(np.int32)).cuda(), b).to_numpy()
        ref = builder.build_soup(torch.from_numpy(soup_of(v4, idx)).cuda(), b).to_numpy()
        check_same_tree(got, ref, f"quads {quads}")


def test_single_and_empty(builder):
    v4 = np.array([[0, 0, 0, 0], [1, 0, 0, 0], [0, 1, 0, 0]], np.float32)
    got = builder.build_mesh(v4, np.array([[0, 1, 2]], np.uint32)).to_numpy()
    ref = oracle.build(soup_of(v4, np.array([[0, 1, 2]])), None)
    check_same_tree(got, ref, "N=1")
    empty = builder.build_mesh(np.zeros((0, 4), np.float32), np.zeros((0, 3), np.uint32))
    assert empty.nodes.shape[0] == 0


def test_bad_index_rejected(builder):
    import lvbh
    from lvbh import _native
    v4, idx = mesh_of(16, 2)
    idx = idx.copy()
    idx[77, 1] = v4.shape[0]
    with pytest.raises(lvbh.LvbhError) as e:
        builder.build_mesh(v4, idx)
    assert e.value.code == _native.EINVAL


def test_trace_through_indexed_leaves(builder):
    import torch
    from test_parity_gpu import make_rays
    v4, idx = mesh_of(256, 7)
    dv = torch.from_numpy(v4).cuda()
    res = builder.build_mesh(dv, torch.from_numpy(idx.view(np.int32)).cuda())
    soup = builder.build_soup(torch.from_numpy(soup_of(v4, idx)).cuda())
    rays = torch.from_numpy(make_rays(1 << 16, seed=9)).cuda()
    pm, tm, sm = builder.trace_mesh(res, dv, rays)
    ps, ts, ss = builder.trace(soup, rays)
    np.testing.assert_array_equal(pm.cpu().numpy(), ps.cpu().numpy())
    np.testing.assert_array_equal(tm.cpu().numpy().view(np.uint32), ts.cpu().numpy().view(np.uint32))
    np.testing.assert_array_equal(sm.cpu().numpy(), ss.cpu().numpy())
    assert (pm >= 0).float().mean().item() > 0.3
