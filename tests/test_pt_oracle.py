"""The path-trace bounce oracle (oracle/pt_oracle.cpp) against independent checks.

sin / cos (the shader leaves their precision to the implementation; the bounce fixes them to a
Cody-Waite reduction and Taylor polynomials) within 2 ulp of the double-precision values, and
the first bounce of an empty scene - every path misses - worked out with numpy float32
arithmetic in the shader's order: baseHash seeds (pathtracer.js:752-756), rand2 (:757-761),
getCameraRay (:720-734) and the miss branch of ptStep (:701-705).
"""
import math

import numpy as np

import oracle

f = np.float32


def ulp_err(got, want):
    want = np.asarray(want, dtype=np.float64)
    return np.abs(got.astype(np.float64) - want) / np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)


def test_sincos_within_two_ulp():
    theta = np.linspace(0.0, 2.0 * math.pi, 1_000_001, dtype=np.float32)
    theta = theta[theta < f(2.0 * math.pi)]
    s, c = oracle.pt_sincos(theta)
    assert ulp_err(s, np.sin(theta.astype(np.float64))).max() <= 2.0
    assert ulp_err(c, np.cos(theta.astype(np.float64))).max() <= 2.0
    s0, c0 = oracle.pt_sincos(np.zeros(1, dtype=np.float32))
    assert s0[0] == 0.0 and c0[0] == 1.0


def base_hash(px, py):
    m = 0xFFFFFFFF
    p2x = (1103515245 * ((px >> 1) ^ py)) & m
    p2y = (1103515245 * ((py >> 1) ^ px)) & m
    h = (1103515245 * (p2x ^ (p2y >> 3))) & m
    return h ^ (h >> 16)


def rand2(seed):
    bx = int(np.array([f(seed + f(1.0))], dtype=np.float32).view(np.uint32)[0])
    by = int(np.array([f(seed + f(2.0))], dtype=np.float32).view(np.uint32)[0])
    n = base_hash(bx, by)
    return f(f(n & 0x7FFFFFFF) / f(2147483648.0)), f(f((n * 48271) & 0xFFFFFFFF & 0x7FFFFFFF) / f(2147483648.0))


def normalize(v):
    ln = f(np.sqrt(f(f(f(v[0] * v[0]) + f(v[1] * v[1])) + f(v[2] * v[2]))))
    return [f(v[0] / ln), f(v[1] / ln), f(v[2] / ln)]


def camera_dir(cx, cy, r, w, h, pos, lat, aspect, sinfov):
    sx = f(f(f(f(cx) + r[0]) / f(w)) * f(2.0)) - f(1.0)
    sy = -(f(f(f(f(cy) + r[1]) / f(h)) * f(2.0)) - f(1.0))
    local = normalize([f(f(aspect * sx) * sinfov), f(1.0), f(sy * sinfov)])
    fw = normalize([f(lat[i] - pos[i]) for i in range(3)])
    right = normalize([fw[1], -fw[0], f(0.0)])
    up = [f(f(right[1] * fw[2]) - f(right[2] * fw[1])), f(f(right[2] * fw[0]) - f(right[0] * fw[2])),
          f(f(right[0] * fw[1]) - f(right[1] * fw[0]))]
    return [f(f(f(right[i] * local[0]) + f(fw[i] * local[1])) + f(up[i] * local[2])) for i in range(3)]


def test_first_bounce_of_an_empty_scene():
    w, h = 7, 5
    pos, lat = [f(3.0), f(0.5), f(0.25)], [f(0.0), f(0.0), f(0.0)]
    out = oracle.pt_step(np.zeros((0, 16), np.uint32), np.zeros((0, 12), np.float32), None, w, h, pos, lat, True)
    aspect, sinfov, _ = oracle.pt_constants(w, h)
    for cy in range(h):
        for cx in range(w):
            seed = f(f(f(base_hash(cx, cy)) / f(4294967296.0)) + f(0.008))
            r = rand2(seed)
            d = camera_dir(cx, cy, r, w, h, pos, lat, aspect, sinfov)
            o4, d4, t4, b4 = (out[k, cy, cx] for k in range(4))
            np.testing.assert_array_equal(o4, np.array(pos + [f(seed + f(2.0))], np.float32))
            np.testing.assert_array_equal(d4, np.array(d + [f(0.0)], np.float32))  # bounces -1 + 1
            np.testing.assert_array_equal(t4, np.array([8, 8, 8, 1], np.float32))  # b = 1 x 8 on a miss
            np.testing.assert_array_equal(b4, np.array([0, 0, 0, 1], np.float32))
    # the next sample starts new paths from the stored seeds and accumulates
    out2 = oracle.pt_step(np.zeros((0, 16), np.uint32), np.zeros((0, 12), np.float32), out, w, h, pos, lat, False)
    np.testing.assert_array_equal(out2[2][..., 3], np.full((h, w), 2, np.float32))
    np.testing.assert_array_equal(out2[2][..., :3], np.full((h, w, 3), 16, np.float32))
    seed2 = out[0][..., 3] + np.float32(2.0)
    np.testing.assert_array_equal(out2[0][..., 3], seed2)


def test_bounce_on_a_floor_stays_finite():
    """A diffuse floor under the camera: paths bounce, the throughput takes pow(.3, 2.2) per
    bounce, roulette ends them after three bounces, every value stays finite."""
    from lvbh import scenes
    tri, bounds = scenes.obj_like_with_floor(2000, seed=5)
    ref = oracle.build(tri, bounds, threads=0)
    w, h = 32, 24
    pos, lat = [0.5, -2.0, 1.5], [0.5, 0.5, 0.3]
    st = None
    for k in range(12):
        st = oracle.pt_step(ref["nodes"], ref["tris"], st, w, h, pos, lat, k == 0)
        assert np.isfinite(st).all()
    b = st[3][..., :3]
    powc = oracle.pt_constants(w, h)[2]
    assert ((b == 0) | (b > 0)).all() and b.max() <= 1.0 / (1.0 - 0.95) * powc + 1e-6
    assert (st[2][..., 3] >= 1).any()
