"""CPU oracle for the LBVH build - TEST INFRASTRUCTURE ONLY.

ctypes wrapper over oracle/liblvbh_oracle.so, the C++ restatement of the reference's WGSL
build (scripts/bvh/kernels/*.js) and traversal (scripts/pathtracer/pathtracer.js).  Only the
tests, the smoke check and the benchmark's CPU-baseline / reference arm use it, as the
checker; the product library never does.

Parity status: unpinned against a run of the reference (it has no tests or golden vectors
and cannot run here); cross-checked against the literal WGSL simulation in
tests/golden/make_golden.py and its committed fixtures.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblvbh_oracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build_lib() -> str:
    """Compile the oracle (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(_HERE, f) for f in ("lvbh_oracle.cpp", "obj_oracle.cpp", "pt_oracle.cpp")]
        if not os.path.exists(_LIB_PATH) or any(
                os.path.exists(f) and os.path.getmtime(f) > os.path.getmtime(_LIB_PATH) for f in srcs):
            build_lib()
        L = ctypes.CDLL(_LIB_PATH)
        vp = ctypes.c_void_p
        u32 = ctypes.c_uint32
        L.oracle_scene_bounds.argtypes = [_f32p, u32, _f32p]
        L.oracle_aabb_zidx.argtypes = [_f32p, u32, _f32p, vp, _u32p, ctypes.c_int]
        L.oracle_radix_sort.argtypes = [_u32p, u32, _i32p, ctypes.c_int]
        L.oracle_radix_tree.argtypes = [_u32p, u32, _i32p, ctypes.c_int]
        L.oracle_up_pass.argtypes = [_i32p, _f32p, _i32p, u32, _u32p, ctypes.c_int]
        L.oracle_canonicalize.argtypes = [_u32p, u32]
        L.oracle_rearrange.argtypes = [_f32p, _i32p, u32, _f32p, ctypes.c_int]
        L.oracle_gather_indexed.argtypes = [_f32p, _u32p, u32, _f32p]
        L.oracle_build.argtypes = [_f32p, u32, vp, ctypes.c_int, vp, vp, vp, vp, vp, vp]
        L.oracle_build.restype = ctypes.c_int
        L.oracle_trace.argtypes = [_u32p, _f32p, u32, _f32p, u32, _i32p, _f32p, _u32p, ctypes.c_int]
        L.oracle_parse_obj.argtypes = [ctypes.c_char_p, ctypes.c_uint64, vp, ctypes.c_uint64,
                                       ctypes.POINTER(ctypes.c_uint64), vp, ctypes.POINTER(ctypes.c_int64)]
        L.oracle_parse_obj.restype = ctypes.c_int
        L.oracle_pt_step.argtypes = [_u32p, _f32p, u32, vp, _f32p, ctypes.POINTER(PtFrame)]
        L.oracle_pt_sincos.argtypes = [_f32p, u32, _f32p, _f32p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def scene_bounds(tri: np.ndarray) -> np.ndarray:
    tri = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 12)
    b = np.empty(6, dtype=np.float32)
    lib().oracle_scene_bounds(tri, tri.shape[0], b)
    return b


def aabb_zidx(tri: np.ndarray, bounds6, threads: int = 1):
    """(aabb (N, 8) float32, keys (N,) uint32) in input order."""
    tri = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 12)
    n = tri.shape[0]
    b = np.ascontiguousarray(bounds6, dtype=np.float32)
    aabb = np.empty((n, 8), dtype=np.float32)
    keys = np.empty(n, dtype=np.uint32)
    lib().oracle_aabb_zidx(tri, n, b, _ptr(aabb), keys, threads)
    return aabb, keys


def radix_sort(keys: np.ndarray, threads: int = 1):
    """(sorted keys, permutation) of the reference's 2-bit x 16-pass stable radix sort."""
    k = np.array(keys, dtype=np.uint32, copy=True)
    perm = np.empty(k.size, dtype=np.int32)
    lib().oracle_radix_sort(k, k.size, perm, threads)
    return k, perm


def radix_tree(sorted_keys: np.ndarray, threads: int = 1) -> np.ndarray:
    k = np.ascontiguousarray(sorted_keys, dtype=np.uint32)
    parents = np.empty(2 * k.size, dtype=np.int32)
    lib().oracle_radix_tree(k, k.size, parents, threads)
    return parents


def up_pass(perm, aabb, parents, threads: int = 1, canonical: bool = True) -> np.ndarray:
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    n = perm.size
    nodes = np.empty((n, 16), dtype=np.uint32)
    lib().oracle_up_pass(perm, np.ascontiguousarray(aabb, dtype=np.float32),
                         np.ascontiguousarray(parents, dtype=np.int32), n, nodes, threads)
    if canonical:
        lib().oracle_canonicalize(nodes, n)
    return nodes


def canonicalize(nodes: np.ndarray) -> np.ndarray:
    nodes = np.array(nodes, dtype=np.uint32, copy=True).reshape(-1, 16)
    lib().oracle_canonicalize(nodes, nodes.shape[0])
    return nodes


def rearrange(tri, perm, threads: int = 1) -> np.ndarray:
    tri = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 12)
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    out = np.empty((perm.size, 12), dtype=np.float32)
    lib().oracle_rearrange(tri, perm, perm.size, out, threads)
    return out


def gather_indexed(xyz, idx3) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    idx3 = np.ascontiguousarray(idx3, dtype=np.uint32).reshape(-1, 3)
    out = np.empty((idx3.shape[0], 12), dtype=np.float32)
    lib().oracle_gather_indexed(xyz, idx3, idx3.shape[0], out)
    return out


def build(tri: np.ndarray, bounds6=None, threads: int = 1) -> dict:
    """The whole build in canonical form: nodes (N, 16) uint32 words, tris (N, 12) float32,
    parents (2N,) int32, leaf_index (N,) uint32, morton (N,) uint32, bounds (6,) float32."""
    tri = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 12)
    n = tri.shape[0]
    out = dict(nodes=np.empty((n, 16), dtype=np.uint32), tris=np.empty((n, 12), dtype=np.float32),
               parents=np.empty(2 * n, dtype=np.int32), leaf_index=np.empty(n, dtype=np.int32),
               morton=np.empty(n, dtype=np.uint32), bounds=np.empty(6, dtype=np.float32))
    b = None if bounds6 is None else np.ascontiguousarray(bounds6, dtype=np.float32)
    rc = lib().oracle_build(tri, n, _ptr(b), threads, _ptr(out["nodes"]), _ptr(out["tris"]),
                            _ptr(out["parents"]), _ptr(out["leaf_index"]), _ptr(out["morton"]),
                            _ptr(out["bounds"]))
    assert rc == 0
    out["leaf_index"] = out["leaf_index"].view(np.uint32)
    return out


def trace(nodes, tris, rays, threads: int = 0):
    """(hit_prim int32, hit_t float32, max_stack uint32) per ray; rays (R, 8) float32."""
    nodes = np.ascontiguousarray(nodes, dtype=np.uint32).reshape(-1, 16)
    tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 12)
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    r = rays.shape[0]
    prim = np.empty(r, dtype=np.int32)
    t = np.empty(r, dtype=np.float32)
    st = np.empty(r, dtype=np.uint32)
    lib().oracle_trace(nodes, tris, tris.shape[0], rays, r, prim, t, st, threads)
    return prim, t, st


class ObjThrows(ValueError):
    """The reference's parseObj throws on this text; .line is the 1-based line of the statement
    (0: a failure after parsing - no model, or a face index naming no vertex)."""

    def __init__(self, line: int):
        super().__init__(f"the reference throws (line {line})")
        self.line = line


def parse_obj(text):
    """OBJ text (str or bytes) -> (tri (N, 12) float32, bounds (6,) float64) as parseObj
    (scripts/obj/parse-obj.js) and build()'s Float32Array produce them, or raises ObjThrows
    where the reference throws."""
    data = text.encode() if isinstance(text, str) else bytes(text)
    n = ctypes.c_uint64()
    line = ctypes.c_int64()
    b = np.empty(6, dtype=np.float64)
    rc = lib().oracle_parse_obj(data, len(data), None, 0, ctypes.byref(n), _ptr(b), ctypes.byref(line))
    if rc != 0:
        raise ObjThrows(int(line.value))
    tri = np.empty((n.value, 12), dtype=np.float32)
    rc = lib().oracle_parse_obj(data, len(data), _ptr(tri), n.value, ctypes.byref(n), _ptr(b),
                                ctypes.byref(line))
    assert rc == 0
    return tri, b


class PtFrame(ctypes.Structure):
    """The bounce's per-frame inputs (OraclePtFrame in pt_oracle.cpp)."""
    _fields_ = [("pos", ctypes.c_float * 3), ("rst", ctypes.c_float), ("lat", ctypes.c_float * 3),
                ("pad", ctypes.c_float), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("aspect", ctypes.c_float), ("sinfov", ctypes.c_float), ("powc", ctypes.c_float),
                ("pad2", ctypes.c_float)]


def pt_constants(width: int, height: int):
    """The constants the reference's shader bakes in: aspect = w / h, sin(.5 * fov * Pi / 180)
    with its argument in float, pow(.3, 2.2), each rounded to float."""
    import math
    f = np.float32
    half_fov = f(f(f(0.5) * f(60.0)) * f(math.pi)) / f(180.0)
    return (f(width / height), f(math.sin(float(half_fov))), f(math.pow(float(f(0.3)), float(f(2.2)))))


def pt_step(nodes, tris, state, width: int, height: int, pos, lat, rst: bool) -> np.ndarray:
    """One sample() of the reference's path tracer (scripts/pathtracer/pathtracer.js:360-392,
    630-772) over a built tree: state (4, height, width, 4) float32 planes o, d, t, b -> the next
    state.  state may be None when rst."""
    nodes = np.ascontiguousarray(nodes).view(np.uint32).reshape(-1)
    tris = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1)
    n = tris.size // 12
    out = np.empty((4, height, width, 4), dtype=np.float32)
    aspect, sinfov, powc = pt_constants(width, height)
    fr = PtFrame((ctypes.c_float * 3)(*pos), 1.0 if rst else 0.0, (ctypes.c_float * 3)(*lat), 0.0,
                 width, height, aspect, sinfov, powc, 0.0)
    sin = None if state is None else np.ascontiguousarray(state, dtype=np.float32)
    lib().oracle_pt_step(nodes, tris, n, _ptr(sin), out, ctypes.byref(fr))
    return out


def pt_sincos(theta):
    theta = np.ascontiguousarray(theta, dtype=np.float32)
    s = np.empty_like(theta)
    c = np.empty_like(theta)
    lib().oracle_pt_sincos(theta, theta.size, s, c)
    return s, c

