"""Seeded synthetic scenes for the LBVH builder.

The reference builds whatever OBJ file is dropped on its page (scripts/main.js:94-136 ->
scripts/obj/parse-obj.js:3-88) and publishes no scene set, so these generators stand in for
it with the shapes, sizes and value distributions of the five build workloads:

  uniform_soup      65,536 triangles, centroids uniform in [0,1]^3, vertex offsets
                    uniform in [-0.005, 0.005]^3 (the small parity workload)
  sphere_mesh       1024 x 1024 quads x 2 = 2,097,152 triangles on a displaced unit
                    sphere, r = 1 + 0.05 * sum_k sin(k theta + phi_k) cos(k psi + chi_k)
  clustered_soup    2^24 triangles, 90 % of the centroids from 64 isotropic Gaussians
                    (means uniform in [0,1]^3, sigma log-uniform in [0.002, 0.05]), 10 %
                    uniform background, vertex offsets uniform in [-0.001, 0.001]^3
  mesh_batch        many independent uniform_soup meshes of log-uniform sizes, each inside
                    its own random box with corners uniform in [-100, 100]^3
  request_sizes     log-uniform request sizes for the build server
  sphere_rays       rays for the sphere: origins uniform on a radius-3 sphere, directions
                    toward uniform points in [-1, 1]^3
  obj_text          an indexed mesh written as the OBJ text an exporter writes (one `o`,
                    `v x y z` with six decimals, `s off`, `f a b c`), the input of the
                    OBJ ingest (parse-obj.js)

All randomness comes from numpy's PCG64 generator seeded by the caller.  Every scene is
returned as the reference's 48-byte triangle layout: float32 array (N, 12), vertices at
columns 0-2, 4-6, 8-10, the pad columns holding 3.1415 as parse-obj.js:55-59 writes them.
"""
from __future__ import annotations

import numpy as np

PAD = np.float32(3.1415)


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def soup_from_vertices(v0: np.ndarray, v1: np.ndarray, v2: np.ndarray, pad=PAD) -> np.ndarray:
    """Pack three (N, 3) vertex arrays into the (N, 12) float32 triangle layout."""
    n = v0.shape[0]
    tri = np.empty((n, 12), dtype=np.float32)
    tri[:, 0:3] = v0
    tri[:, 4:7] = v1
    tri[:, 8:11] = v2
    tri[:, 3] = pad
    tri[:, 7] = pad
    tri[:, 11] = pad
    return tri


def indexed_from_soup(tri: np.ndarray):
    """Indexed form (float32 xyz (3N, 3), uint32 idx3 (N, 3)) of a soup: triple (3i, 3i+1, 3i+2)."""
    n = tri.shape[0]
    xyz = np.empty((3 * n, 3), dtype=np.float32)
    xyz[0::3] = tri[:, 0:3]
    xyz[1::3] = tri[:, 4:7]
    xyz[2::3] = tri[:, 8:11]
    idx3 = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return xyz, idx3


def uniform_soup(n: int = 65_536, seed: int = 0, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                 half_offset: float = 0.005) -> np.ndarray:
    """Centroids uniform in the box [lo, hi]; each vertex = centroid + uniform offset in
    [-half_offset, half_offset]^3 scaled by the box extent (float32)."""
    rng = _rng(seed)
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    ext = hi - lo
    c = lo + rng.random((n, 3)) * ext
    vs = [(c + (rng.random((n, 3)) * 2.0 - 1.0) * half_offset * ext).astype(np.float32)
          for _ in range(3)]
    return soup_from_vertices(*vs)


def sphere_mesh(quads: int = 1024, seed: int = 1, indexed: bool = False):
    """A quads x quads grid over (theta, psi), two triangles per quad, mapped onto a sphere
    with radius 1 + 0.05 * sum_{k=1..8} sin(k theta + phi_k) cos(k psi + chi_k)."""
    rng = _rng(seed)
    phi = rng.random(8) * 2.0 * np.pi
    chi = rng.random(8) * 2.0 * np.pi
    th = np.linspace(0.0, np.pi, quads + 1)              # polar angle, poles included
    ps = np.linspace(0.0, 2.0 * np.pi, quads + 1)        # azimuth, seam duplicated
    T, P = np.meshgrid(th, ps, indexing="ij")
    r = np.ones_like(T)
    for k in range(1, 9):
        r += 0.05 * np.sin(k * T + phi[k - 1]) * np.cos(k * P + chi[k - 1])
    xyz = np.stack([r * np.sin(T) * np.cos(P), r * np.sin(T) * np.sin(P), r * np.cos(T)],
                   axis=-1).reshape(-1, 3).astype(np.float32)
    g = quads + 1
    i, j = np.meshgrid(np.arange(quads), np.arange(quads), indexing="ij")
    a = (i * g + j).ravel()
    b = a + 1
    c = a + g
    d = c + 1
    idx3 = np.empty((2 * a.size, 3), dtype=np.uint32)
    idx3[0::2] = np.stack([a, c, b], axis=1)
    idx3[1::2] = np.stack([b, c, d], axis=1)
    if indexed:
        return xyz, idx3
    return soup_from_vertices(xyz[idx3[:, 0]], xyz[idx3[:, 1]], xyz[idx3[:, 2]])


def clustered_soup(n: int = 1 << 24, seed: int = 2, clusters: int = 64,
                   background: float = 0.10, half_offset: float = 0.001) -> np.ndarray:
    """Centroids from a mixture of isotropic Gaussians plus a uniform background."""
    rng = _rng(seed)
    means = rng.random((clusters, 3))
    sig = np.exp(rng.uniform(np.log(0.002), np.log(0.05), clusters))
    nb = int(round(n * background))
    nc = n - nb
    which = rng.integers(0, clusters, nc)
    c = np.empty((n, 3), dtype=np.float64)
    c[:nc] = means[which] + rng.standard_normal((nc, 3)) * sig[which, None]
    c[nc:] = rng.random((nb, 3))
    c = c[rng.permutation(n)]
    vs = []
    for _ in range(3):
        off = rng.random((n, 3), dtype=np.float32) * np.float32(2.0) - np.float32(1.0)
        vs.append((c.astype(np.float32) + off * np.float32(half_offset)))
    return soup_from_vertices(*vs)


def mesh_batch_sizes(count: int = 4096, lo: int = 64, hi: int = 262_144, seed: int = 3) -> np.ndarray:
    """Per-mesh triangle counts, log-uniform in [lo, hi]."""
    rng = _rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count))).astype(np.int64).clip(lo, hi)


def mesh_batch(count: int = 4096, lo: int = 64, hi: int = 262_144, seed: int = 3):
    """`count` independent uniform_soup meshes of log-uniform sizes, each in its own box with
    corners uniform in [-100, 100]^3.  Returns (soup (sum N, 12), offsets (count + 1,) int64)."""
    sizes = mesh_batch_sizes(count, lo, hi, seed)
    rng = _rng(seed + 1)
    corners = rng.uniform(-100.0, 100.0, (count, 2, 3))
    offsets = np.zeros(count + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(sizes)
    soup = np.empty((int(offsets[-1]), 12), dtype=np.float32)
    for m in range(count):
        lo_c = corners[m].min(axis=0)
        hi_c = corners[m].max(axis=0)
        soup[offsets[m]:offsets[m + 1]] = uniform_soup(int(sizes[m]), seed=seed * 100_003 + m,
                                                       lo=lo_c, hi=hi_c)
    return soup, offsets


def sphere_rays(n: int = 1 << 20, seed: int = 11, radius: float = 3.0) -> np.ndarray:
    """(n, 8) float32 rays {ox, oy, oz, 0, dx, dy, dz, 0}: origins uniform on a sphere of the
    given radius, unit directions toward points uniform in [-1, 1]^3."""
    rng = _rng(seed)
    o = rng.standard_normal((n, 3))
    o = o / np.linalg.norm(o, axis=1, keepdims=True) * radius
    d = rng.uniform(-1.0, 1.0, (n, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros((n, 8), dtype=np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    return rays


def request_sizes(count: int = 100_000, lo: int = 1024, hi: int = 4_194_304, seed: int = 4) -> np.ndarray:
    """Build-request sizes, log-uniform in [lo, hi]."""
    rng = _rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), count))).astype(np.int64).clip(lo, hi)


def obj_like_with_floor(n: int = 4096, seed: int = 5):
    """A uniform soup plus the two floor triangles parse-obj.js:66-78 appends at +-10000 and
    z_min + .01 (after its y/z swap), with the host bounds computed from the model's vertices
    only, as parse-obj.js:27-53 does.  Returns (soup, bounds6) - the floor lies outside the
    bounds, which drives quantised coordinates past 1023 exactly as in the reference."""
    tri = uniform_soup(n, seed)
    mn = tri[:, [0, 1, 2]].min(axis=0)
    mn = np.minimum(mn, tri[:, [4, 5, 6]].min(axis=0))
    mn = np.minimum(mn, tri[:, [8, 9, 10]].min(axis=0))
    mx = tri[:, [0, 1, 2]].max(axis=0)
    mx = np.maximum(mx, tri[:, [4, 5, 6]].max(axis=0))
    mx = np.maximum(mx, tri[:, [8, 9, 10]].max(axis=0))
    h = np.float32(mn[2] + np.float32(0.01))
    s = np.float32(10000.0)
    floor = np.array([[-s, -s, h, PAD, s, -s, h, PAD, -s, s, h, PAD],
                      [s, -s, h, PAD, s, s, h, PAD, -s, s, h, PAD]], dtype=np.float32)
    bounds = np.concatenate([mn, mx]).astype(np.float32)
    return np.concatenate([tri, floor]), bounds


def obj_text(xyz: np.ndarray, idx3: np.ndarray, name: str = "mesh") -> bytes:
    """Indexed mesh (V, 3) + (F, 3) 0-based -> OBJ text (UTF-8 bytes): a comment line, `o name`,
    one `v` line per vertex with six decimals, `s off`, one `f` line per triangle (1-based)."""
    head = f"# synthetic mesh: {xyz.shape[0]} vertices, {idx3.shape[0]} faces\no {name}\n"
    v = "\n".join("v %.6f %.6f %.6f" % (float(a), float(b), float(c)) for a, b, c in xyz.tolist())
    f = "\n".join("f %d %d %d" % (a + 1, b + 1, c + 1) for a, b, c in idx3.tolist())
    return (head + v + "\ns off\n" + f + "\n").encode()

