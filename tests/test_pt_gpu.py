"""Path-trace bounce on the GPU (lvbh_pt_sample, through the C ABI) against the oracle.

Every word of the four state planes (origin + seed, direction + bounce count, accumulated
radiance + sample count, throughput) must equal the oracle's after every sample, over many
samples with ping-pong buffers and a reset in between, on trees built by the device builder.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def run_both(builder, tri, bounds, w, h, steps, reset_at=(), rot=0.0):
    import torch
    import lvbh
    res = builder.build_soup(torch.from_numpy(tri).cuda(), bounds)
    ref = res.to_numpy()
    model = bounds if bounds is not None else ref["bounds"]
    pos, lat = lvbh.camera([float(x) for x in model], rot)
    bufs = [torch.zeros((4, h, w, 4), dtype=torch.float32, device="cuda") for _ in range(2)]
    st = None
    for k in range(steps):
        rst = k == 0 or k in reset_at
        src, dst = bufs[k % 2], bufs[(k + 1) % 2]
        builder.pt_sample(res, None if rst else src, dst, w, h, pos, lat, reset=rst)
        st = oracle.pt_step(ref["nodes"], ref["tris"], None if rst else st, w, h, pos, lat, rst)
        got = dst.cpu().numpy()
        bad = np.nonzero(got.view(np.uint32) != st.view(np.uint32))
        assert bad[0].size == 0, f"sample {k}: {bad[0].size} words differ, first at {[b[:4] for b in bad]}"
    return st


def test_floor_scene_many_samples(builder):
    from lvbh import scenes
    tri, bounds = scenes.obj_like_with_floor(5000, seed=5)
    st = run_both(builder, tri, bounds, 96, 64, 24, reset_at=(13,))
    assert (st[2][..., 3] > 0).all()


def test_sphere_and_rotation(builder):
    from lvbh import scenes
    tri = scenes.sphere_mesh(96, seed=1)
    run_both(builder, tri, None, 80, 48, 10, rot=np.pi / 4)


def test_empty_scene_and_odd_sizes(builder):
    run_both(builder, np.zeros((0, 12), np.float32), np.array([0, 0, 0, 1, 1, 1], np.float32), 13, 7, 3)


def test_bad_arguments(builder):
    import torch
    import lvbh
    from lvbh import _native
    res = builder.build_soup(torch.zeros((4, 12), dtype=torch.float32, device="cuda"))
    out = torch.zeros((4, 8, 8, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError):
        builder.pt_sample(res, None, out[:, :4], 8, 8, [1, 1, 1], [0, 0, 0], reset=True)
    with pytest.raises(lvbh.LvbhError) as e:
        builder.pt_sample(res, None, out, 8, 8, [1, 1, 1], [0, 0, 0], reset=False)
    assert e.value.code == _native.EINVAL
