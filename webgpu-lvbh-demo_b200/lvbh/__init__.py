"""B200-native LBVH builder - Python host side of the C ABI in include/lvbh.h.

Mirrors the reference's build entry (scripts/bvh/build-bvh.js):

    BVH = initBVHBuild(device)                                   # build-bvh.js:1-10
    out = BVH.build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS)           # build-bvh.js:12-66
    out["BVH_BUFFER"], out["O_TRIANGLE_BUFFER"]

with the same argument meaning: TRI_ARRAY holds 12 floats per triangle (the pad slot is
ignored), MODEL_BOUNDS is {"min": [x, y, z], "max": [x, y, z]} (parse-obj.js:80-87) or None to
reduce the scene box on the device.  As in the reference, a TRI_ARRAY longer than
12 * NUM_TRIS is an error (Float32Array.set throws a RangeError, build-bvh.js:20) and a shorter
one leaves the remaining floats zero.  Results stay on the GPU as torch tensors; the reference
returns GPU buffers the same way (build-bvh.js:65).

torch provides device memory and streams only; every byte of the build is computed by the
sm_100a kernels in liblvbh.so.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native
from ._native import (ASYNC, AUTOTUNE, INPUT_HOST, NO_GRAPH, OUT_CALLER, PROFILE, STAGE_NAMES,
                      LvbhError, version)

__all__ = ["initBVHBuild", "BVHBuilder", "BuildResult", "BatchResult", "LvbhError", "ObjError",
           "version", "trace", "parseObj"]


def _torch():
    import torch
    return torch


def _stream_ptr(stream, device):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream(device)
    return ctypes.c_void_p(stream.cuda_stream)


def bounds_from_model(model_bounds) -> Optional[np.ndarray]:
    """MODEL_BOUNDS ({min, max} dict, 6 floats, or None) -> float32[6] or None."""
    if model_bounds is None:
        return None
    if isinstance(model_bounds, dict):
        b = list(model_bounds["min"]) + list(model_bounds["max"])
    else:
        b = list(np.asarray(model_bounds, dtype=np.float64).ravel())
    if len(b) != 6:
        raise ValueError("MODEL_BOUNDS needs 3 min and 3 max values")
    return np.asarray(b, dtype=np.float32)  # DataView.setFloat32 rounding (aabb-z-idx.js:116-122)


def soup_from_tri_array(tri_array, num_tris: int):
    """TRI_ARRAY -> (N, 12) float32 host array or CUDA tensor, with the reference's length rule."""
    torch = _torch()
    need = 12 * int(num_tris)
    if isinstance(tri_array, torch.Tensor):
        t = tri_array.reshape(-1)
        if t.numel() > need:
            raise ValueError(f"RangeError: TRI_ARRAY holds {t.numel()} floats, NUM_TRIS*12 = {need}")
        if t.dtype != torch.float32:
            t = t.to(torch.float32)
        if t.numel() < need:
            t = torch.cat([t, torch.zeros(need - t.numel(), dtype=torch.float32, device=t.device)])
        return t.contiguous().reshape(int(num_tris), 12)
    a = np.asarray(tri_array, dtype=np.float32).reshape(-1)
    if a.size > need:
        raise ValueError(f"RangeError: TRI_ARRAY holds {a.size} floats, NUM_TRIS*12 = {need}")
    if a.size < need:
        a = np.concatenate([a, np.zeros(need - a.size, dtype=np.float32)])
    return np.ascontiguousarray(a).reshape(int(num_tris), 12)


@dataclass
class BuildResult:
    """Device-resident result.  nodes: int32 (N, 16) BVHNode words (box words are float32 bits,
    view with .view(torch.float32)); tris: float32 (N, 12); parents: int32 (2N,);
    leaf_index: int32 (N,) (the reference's IDX_BUFFER); morton: int32 (N,) key bits;
    bounds: float32 (6,) quantisation box; stage_ms: per-stage device times when profiled."""
    nodes: object
    tris: object
    parents: object
    leaf_index: object
    morton: object
    bounds: np.ndarray
    stage_ms: Optional[dict] = None

    def as_reference(self) -> dict:
        """{BVH_BUFFER, O_TRIANGLE_BUFFER} as the reference's build() returns them."""
        return {"BVH_BUFFER": self.nodes, "O_TRIANGLE_BUFFER": self.tris}

    def to_numpy(self) -> dict:
        return {"nodes": self.nodes.cpu().numpy().view(np.uint32),
                "tris": self.tris.cpu().numpy(),
                "parents": self.parents.cpu().numpy(),
                "leaf_index": self.leaf_index.cpu().numpy().view(np.uint32),
                "morton": self.morton.cpu().numpy().view(np.uint32),
                "bounds": self.bounds.copy()}


@dataclass
class BatchResult(BuildResult):
    """Result of a batched build: the concatenated per-mesh buffers plus the mesh offsets
    (int64, num_meshes + 1) and each mesh's quantisation box seg_bounds (float32, (M, 6))."""
    offsets: Optional[np.ndarray] = None
    seg_bounds: Optional[np.ndarray] = None

    def mesh(self, i: int) -> BuildResult:
        """Views of mesh i's slice - a standalone BVH of that mesh, identical to building it
        alone with build_soup."""
        a, b = int(self.offsets[i]), int(self.offsets[i + 1])
        return BuildResult(nodes=self.nodes[a:b], tris=self.tris[a:b],
                           parents=self.parents[2 * a:2 * b], leaf_index=self.leaf_index[a:b],
                           morton=self.morton[a:b], bounds=self.seg_bounds[i].copy())


def empty_outputs(n: int, device, mesh: bool = False):
    """Result buffers of an n-triangle build; mesh: the indexed leaf format's tris (n, 3) uint32."""
    torch = _torch()
    tris = (torch.empty((n, 3), dtype=torch.int32, device=device) if mesh
            else torch.empty((n, 12), dtype=torch.float32, device=device))
    return dict(nodes=torch.empty((n, 16), dtype=torch.int32, device=device), tris=tris,
                parents=torch.empty(2 * n, dtype=torch.int32, device=device),
                leaf_index=torch.empty(n, dtype=torch.int32, device=device),
                morton=torch.empty(n, dtype=torch.int32, device=device))


def _result_struct(outs, n) -> _native.Result:
    r = _native.Result()
    r.num_tris = n
    r.num_nodes = n
    for k in ("nodes", "tris", "parents", "leaf_index", "morton"):
        setattr(r, k, outs[k].data_ptr() if n else None)
    return r


class BVHBuilder:
    """One library context bound to a CUDA device (initBVHBuild(device), build-bvh.js:1-10)."""

    def __init__(self, device=0, reserve_tris: int = 0):
        torch = _torch()
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        cfg = _native.Config(device=self.device.index or 0, reserve_tris=int(reserve_tris))
        ctx = ctypes.c_void_p()
        rc = _native.lib.lvbh_create(ctypes.byref(ctx), ctypes.byref(cfg))
        if rc != _native.OK:
            raise LvbhError(rc, "lvbh_create failed")
        self._ctx = ctx
        self._pending = None

    def close(self):
        if getattr(self, "_ctx", None):
            # at interpreter exit the module's globals may already be gone
            lib = getattr(_native, "lib", None) if _native is not None else None
            if lib is not None:
                lib.lvbh_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    @property
    def ctx(self):
        return self._ctx

    # -- reference-shaped entry -------------------------------------------------------------
    def build(self, TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS=None) -> dict:  # noqa: N803
        """build(TRI_ARRAY, NUM_TRIS, MODEL_BOUNDS) -> {BVH_BUFFER, O_TRIANGLE_BUFFER, ...}."""
        res = self.build_soup(soup_from_tri_array(TRI_ARRAY, NUM_TRIS), bounds_from_model(MODEL_BOUNDS))
        out = res.as_reference()
        out.update(PARENT_BUFFER=res.parents, IDX_BUFFER=res.leaf_index, Z_IDX_BUFFER=res.morton,
                   BOUNDS=res.bounds)
        return out

    # -- full-control entries ---------------------------------------------------------------
    def build_soup(self, tri, bounds=None, outputs=None, stream=None, sync=True, profile=False,
                   graph=True) -> BuildResult:
        """tri: (N, 12) float32 numpy array (host, copied inside the call) or CUDA tensor."""
        torch = _torch()
        host = not isinstance(tri, torch.Tensor)
        if host:
            tri = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 12)
            n = tri.shape[0]
            ptr = tri.ctypes.data_as(ctypes.c_void_p)
        else:
            if tri.device.type != "cuda":
                tri = tri.to(self.device)
            tri = tri.contiguous().reshape(-1, 12)
            if tri.dtype != torch.float32:
                raise TypeError("device triangle soup must be float32")
            n = tri.shape[0]
            ptr = ctypes.c_void_p(tri.data_ptr())
        flags = OUT_CALLER | (INPUT_HOST if host else 0) | (0 if sync else ASYNC) \
            | (PROFILE if profile else 0) | (0 if graph else NO_GRAPH)
        return self._run(_native.lib.lvbh_build_soup, (ptr, n), n, bounds, flags, outputs,
                         stream, sync, profile, keep=(tri,))

    def build_indexed(self, xyz, idx3, bounds=None, outputs=None, stream=None, sync=True,
                      profile=False) -> BuildResult:
        """xyz: (V, 3) float32, idx3: (N, 3) uint32 - both host arrays or both CUDA tensors."""
        torch = _torch()
        host = not isinstance(xyz, torch.Tensor)
        if host:
            xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
            idx3 = np.ascontiguousarray(idx3, dtype=np.uint32).reshape(-1, 3)
            pv, pi = xyz.ctypes.data_as(ctypes.c_void_p), idx3.ctypes.data_as(ctypes.c_void_p)
        else:
            xyz = xyz.contiguous().reshape(-1, 3)
            idx3 = idx3.contiguous().reshape(-1, 3)
            pv, pi = ctypes.c_void_p(xyz.data_ptr()), ctypes.c_void_p(idx3.data_ptr())
        n, nv = idx3.shape[0], xyz.shape[0]
        flags = OUT_CALLER | (INPUT_HOST if host else 0) | (0 if sync else ASYNC) \
            | (PROFILE if profile else 0)
        return self._run(_native.lib.lvbh_build_indexed, (pv, nv, pi, n), n, bounds, flags,
                         outputs, stream, sync, profile, keep=(xyz, idx3))

    def build_mesh(self, verts4, idx3, bounds=None, outputs=None, stream=None, sync=True,
                   profile=False) -> BuildResult:
        """The indexed leaf format (lvbh_build_mesh): verts4 (V, 4) float32 rows {x, y, z, pad},
        idx3 (N, 3) uint32 - both host arrays or both CUDA tensors.  The result's tris are the
        (N, 3) vertex indices of each sorted leaf (int32 tensor holding uint32 values)."""
        torch = _torch()
        host = not isinstance(verts4, torch.Tensor)
        if host:
            verts4 = np.ascontiguousarray(verts4, dtype=np.float32).reshape(-1, 4)
            idx3 = np.ascontiguousarray(idx3, dtype=np.uint32).reshape(-1, 3)
            pv, pi = verts4.ctypes.data_as(ctypes.c_void_p), idx3.ctypes.data_as(ctypes.c_void_p)
        else:
            verts4 = verts4.contiguous().reshape(-1, 4)
            idx3 = idx3.contiguous().reshape(-1, 3)
            pv, pi = ctypes.c_void_p(verts4.data_ptr()), ctypes.c_void_p(idx3.data_ptr())
        n, nv = idx3.shape[0], verts4.shape[0]
        flags = OUT_CALLER | (INPUT_HOST if host else 0) | (0 if sync else ASYNC) \
            | (PROFILE if profile else 0)
        if outputs is None:
            outputs = empty_outputs(n, self.device, mesh=True)
        return self._run(_native.lib.lvbh_build_mesh, (pv, nv, pi, n), n, bounds, flags,
                         outputs, stream, sync, profile, keep=(verts4, idx3))

    def trace_mesh(self, res: BuildResult, verts4, rays, stream=None):
        """lvbh_trace over the indexed leaf format: res from build_mesh, verts4 (V, 4) float32
        CUDA tensor.  Returns (hit_prim int32, hit_t float32, max_stack int32)."""
        torch = _torch()
        rays = rays.contiguous().reshape(-1, 8)
        verts4 = verts4.contiguous().reshape(-1, 4)
        nr = rays.shape[0]
        prim = torch.empty(nr, dtype=torch.int32, device=self.device)
        t = torch.empty(nr, dtype=torch.float32, device=self.device)
        st = torch.empty(nr, dtype=torch.int32, device=self.device)
        n = res.tris.shape[0]
        rc = _native.lib.lvbh_trace_mesh(self._ctx, ctypes.c_void_p(res.nodes.data_ptr() if n else 0),
                                         ctypes.c_void_p(res.tris.data_ptr() if n else 0),
                                         ctypes.c_void_p(verts4.data_ptr() if n else 0), verts4.shape[0], n,
                                         ctypes.c_void_p(rays.data_ptr()), nr, ctypes.c_void_p(prim.data_ptr()),
                                         ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(st.data_ptr()),
                                         _stream_ptr(stream, self.device))
        _native.check(self._ctx, rc)
        return prim, t, st

    def build_batched(self, tri, offsets, seg_bounds=None, outputs=None, stream=None, sync=True,
                      profile=False, graph=True, autotune=False) -> BatchResult:
        """Many meshes in one build.  tri: (sum N, 12) float32 host array or CUDA tensor with
        the meshes end to end; offsets: num_meshes + 1 triangle offsets (offsets[0] = 0);
        seg_bounds: (M, 6) float32 per-mesh MODEL_BOUNDS or None (each mesh's own box)."""
        torch = _torch()
        offs = np.ascontiguousarray(offsets, dtype=np.int64).ravel()
        if offs.size < 1 or offs[0] != 0 or np.any(np.diff(offs) < 0) or offs[-1] > _native.MAX_TRIS:
            raise ValueError("offsets must start at 0, be non-decreasing and end <= 2^29")
        m = offs.size - 1
        offs32 = offs.astype(np.uint32)
        host = not isinstance(tri, torch.Tensor)
        if host:
            tri = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 12)
            ptr = tri.ctypes.data_as(ctypes.c_void_p)
        else:
            if tri.device.type != "cuda":
                tri = tri.to(self.device)
            tri = tri.contiguous().reshape(-1, 12)
            if tri.dtype != torch.float32:
                raise TypeError("device triangle soup must be float32")
            ptr = ctypes.c_void_p(tri.data_ptr())
        n = int(offs[-1])
        if tri.shape[0] != n:
            raise ValueError(f"soup holds {tri.shape[0]} triangles, offsets end at {n}")
        if self._pending is not None:
            self.sync()
        outs = outputs if outputs is not None else empty_outputs(n, self.device)
        r = _result_struct(outs, n)
        sb = None if seg_bounds is None else np.ascontiguousarray(seg_bounds, dtype=np.float32).reshape(m, 6)
        bout = np.zeros((m, 6), dtype=np.float32)
        flags = OUT_CALLER | (INPUT_HOST if host else 0) | (0 if sync else ASYNC) \
            | (PROFILE if profile else 0) | (0 if graph else NO_GRAPH) | (AUTOTUNE if autotune else 0)
        rc = _native.lib.lvbh_build_batched(
            self._ctx, ptr, offs32.ctypes.data_as(ctypes.c_void_p), m,
            None if sb is None else sb.ctypes.data_as(ctypes.c_void_p),
            bout.ctypes.data_as(ctypes.c_void_p), flags, ctypes.byref(r),
            _stream_ptr(stream, self.device))
        res = BatchResult(bounds=np.zeros(6, np.float32), offsets=offs, seg_bounds=bout, **outs)
        if rc != _native.OK:
            _native.check(self._ctx, rc)
        if sync:
            if profile:
                res.stage_ms = self.stage_times()
        else:
            self._pending = (r, res, (tri, offs32, sb, bout), profile)
        return res

    def set_tunables(self, digit_bits=None, tree_block=None, tree_ctas_per_sm=0):
        """Force the batched-build tunables (digit_bits 10 or 8, tree_block 256 or 128);
        no arguments = back to LVBH_AUTOTUNE / the defaults."""
        if digit_bits is None and tree_block is None:
            _native.check(self._ctx, _native.lib.lvbh_set_tunables(self._ctx, None))
            return
        t = _native.Tunables(digit_bits=digit_bits or 10, tree_block=tree_block or 256,
                             tree_ctas_per_sm=tree_ctas_per_sm)
        _native.check(self._ctx, _native.lib.lvbh_set_tunables(self._ctx, ctypes.byref(t)))

    def tunables(self) -> dict:
        """The tunables of the last batched build, and the candidates' times when it tuned."""
        t = _native.Tunables()
        ms = (ctypes.c_float * 4)()
        nc = ctypes.c_uint32()
        _native.check(self._ctx, _native.lib.lvbh_get_tunables(self._ctx, ctypes.byref(t), ms,
                                                               ctypes.byref(nc)))
        return {"digit_bits": t.digit_bits, "tree_block": t.tree_block,
                "tree_ctas_per_sm": t.tree_ctas_per_sm,
                "candidates_ms": [float(x) for x in ms[:nc.value]]}

    def _run(self, fn, head, n, bounds, flags, outputs, stream, sync, profile, keep):
        if self._pending is not None:
            self.sync()
        outs = outputs if outputs is not None else empty_outputs(n, self.device)
        r = _result_struct(outs, n)
        b = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float32).reshape(6)
        bp = None if b is None else b.ctypes.data_as(ctypes.c_void_p)
        sp = _stream_ptr(stream, self.device)
        rc = fn(self._ctx, *head, bp, flags, ctypes.byref(r), sp)
        res = BuildResult(bounds=np.zeros(6, np.float32), **outs)
        if rc != _native.OK:
            _native.check(self._ctx, rc)
        if sync:
            res.bounds = np.array(r.bounds[:], dtype=np.float32)
            if profile:
                res.stage_ms = self.stage_times()
        else:
            self._pending = (r, res, keep, profile)
        return res

    def sync(self):
        """Wait for an asynchronous build and raise its device-side status."""
        if self._pending is None:
            return
        r, res, _, profile = self._pending
        self._pending = None
        _native.check(self._ctx, _native.lib.lvbh_sync(self._ctx))
        if not isinstance(res, BatchResult):
            res.bounds = np.array(r.bounds[:], dtype=np.float32)
        if profile:
            res.stage_ms = self.stage_times()

    def stage_times(self) -> dict:
        arr = (ctypes.c_float * _native.NUM_STAGES)()
        _native.check(self._ctx, _native.lib.lvbh_stage_times(self._ctx, arr))
        return dict(zip(STAGE_NAMES, [float(x) for x in arr]))

    def trace(self, res: BuildResult, rays, stream=None):
        """Closest-hit traversal (scripts/pathtracer/pathtracer.js:495-628) of rays (R, 8)
        float32 CUDA tensor -> (hit_prim int32, hit_t float32, max_stack int32)."""
        torch = _torch()
        rays = rays.contiguous().reshape(-1, 8)
        nr = rays.shape[0]
        prim = torch.empty(nr, dtype=torch.int32, device=self.device)
        t = torch.empty(nr, dtype=torch.float32, device=self.device)
        st = torch.empty(nr, dtype=torch.int32, device=self.device)
        n = res.tris.shape[0]
        rc = _native.lib.lvbh_trace(self._ctx, ctypes.c_void_p(res.nodes.data_ptr() if n else 0),
                                    ctypes.c_void_p(res.tris.data_ptr() if n else 0), n,
                                    ctypes.c_void_p(rays.data_ptr()), nr,
                                    ctypes.c_void_p(prim.data_ptr()), ctypes.c_void_p(t.data_ptr()),
                                    ctypes.c_void_p(st.data_ptr()), _stream_ptr(stream, self.device))
        _native.check(self._ctx, rc)
        return prim, t, st


    def pt_sample(self, res: BuildResult, state_in, state_out, width: int, height: int, pos, lat,
                  reset: bool = False, stream=None):
        """One sample() of the reference's path tracer (pathtracer.js:360-392): every pixel's
        path advances one bounce through the built tree.  state_in / state_out: (4, height,
        width, 4) float32 CUDA tensors, planes o, d, t, b (state_in unread when reset)."""
        for st in (state_in, state_out):
            if st is not None and (tuple(st.shape) != (4, height, width, 4) or not st.is_contiguous()):
                raise ValueError("state must be a contiguous (4, height, width, 4) float32 tensor")
        fr = _native.PtFrame((ctypes.c_float * 3)(*[float(x) for x in pos]), 1.0 if reset else 0.0,
                             (ctypes.c_float * 3)(*[float(x) for x in lat]), 0.0)
        n = res.tris.shape[0]
        rc = _native.lib.lvbh_pt_sample(self._ctx, ctypes.c_void_p(res.nodes.data_ptr() if n else 0),
                                        ctypes.c_void_p(res.tris.data_ptr() if n else 0), n,
                                        ctypes.c_void_p(state_in.data_ptr() if state_in is not None else 0),
                                        ctypes.c_void_p(state_out.data_ptr()), width, height, ctypes.byref(fr),
                                        _stream_ptr(stream, self.device))
        _native.check(self._ctx, rc)
        return state_out

    def parse_obj(self, text, stream=None) -> dict:
        """parseObj(file) (scripts/obj/parse-obj.js:3-88) on the GPU.

        text: the file's bytes (bytes, str as UTF-8, a uint8 numpy array, or a uint8 CUDA
        tensor).  Returns {"NUM_TRIS", "TRI_ARR", "BOUNDS"} as the reference does, TRI_ARR as a
        (NUM_TRIS, 12) float32 CUDA tensor (pad 3.1415, floor included) and BOUNDS as
        {"min": [x, y, z], "max": [x, y, z]} doubles.  Where the reference throws, raises
        ObjError with .line (1-based; 0 for a failure found after parsing).
        """
        torch = _torch()
        keep = None
        flags = 0
        if isinstance(text, torch.Tensor):
            if not text.is_cuda:
                text = text.numpy()
            else:
                keep = text.contiguous().view(torch.uint8).reshape(-1)
                ptr, nbytes = keep.data_ptr(), keep.numel()
        if keep is None:
            if isinstance(text, str):
                text = text.encode("utf-8")
            keep = np.ascontiguousarray(np.frombuffer(text, dtype=np.uint8) if isinstance(text, (bytes, bytearray))
                                        else np.asarray(text, dtype=np.uint8).reshape(-1))
            ptr, nbytes = keep.ctypes.data, keep.size
            flags = INPUT_HOST
        tri = ctypes.c_void_p()
        n = ctypes.c_uint32()
        b6 = (ctypes.c_double * 6)()
        line = ctypes.c_uint64()
        rc = _native.lib.lvbh_parse_obj(self._ctx, ctypes.c_void_p(ptr if nbytes else 0), nbytes, flags,
                                        ctypes.byref(tri), ctypes.byref(n), b6, ctypes.byref(line),
                                        _stream_ptr(stream, self.device))
        if rc == _native.EPARSE:
            raise ObjError(int(line.value), _native.lib.lvbh_last_error(self._ctx).decode())
        _native.check(self._ctx, rc)
        soup = _device_floats(tri.value, n.value * 12, self.device).clone().reshape(n.value, 12)
        return {"NUM_TRIS": n.value, "TRI_ARR": soup,
                "BOUNDS": {"min": [b6[0], b6[1], b6[2]], "max": [b6[3], b6[4], b6[5]]}}


class ObjError(LvbhError):
    """The OBJ text is one the reference's parser throws on."""

    def __init__(self, line: int, message: str):
        super().__init__(_native.EPARSE, message)
        self.line = line


class _DeviceArray:
    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 3}


def _device_floats(ptr, count, device):
    """A float32 CUDA tensor viewing `count` floats at device address `ptr` (no copy)."""
    torch = _torch()
    if count == 0:
        return torch.zeros(0, dtype=torch.float32, device=device)
    return torch.as_tensor(_DeviceArray(ptr, count), device=device)


def initBVHBuild(device=0) -> BVHBuilder:  # noqa: N802
    """initBVHBuild(device) -> object with .build (scripts/bvh/build-bvh.js:1-10)."""
    return BVHBuilder(device)


def trace(builder: BVHBuilder, res: BuildResult, rays):
    return builder.trace(res, rays)


def parseObj(builder: BVHBuilder, file) -> dict:  # noqa: N802
    """parseObj(file) (scripts/obj/parse-obj.js:3-88) on the builder's GPU."""
    return builder.parse_obj(file)


def camera(bounds, rot: float = 0.0):
    """The path tracer's camera for a model (initPathTracer, pathtracer.js:5-23, rotateView
    :418-426): look at the box centre from 1.5 x its largest extent away, rotated by `rot` about
    z.  bounds: {"min", "max"} or 6 numbers.  Returns (pos, lat) as float lists."""
    import math
    b = list(bounds["min"]) + list(bounds["max"]) if isinstance(bounds, dict) else [float(x) for x in bounds]
    dist = 1.5 * max(max(b[3] - b[0], b[4] - b[1]), b[5] - b[2])
    lat = [(b[0] + b[3]) * .5, (b[1] + b[4]) * .5, (b[2] + b[5]) * .5]
    pos = [lat[0] + math.cos(rot) * dist, lat[1] + math.sin(rot) * dist, lat[2]]
    return pos, lat

