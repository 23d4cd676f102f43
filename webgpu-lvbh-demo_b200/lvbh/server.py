"""Build server: continuous batching of build requests on one GPU (C ABI lvbh_server_*).

    srv = Server(device=0, hbm_budget=96 << 30)
    t = srv.submit(tri)                 # CUDA tensor, or host array / pinned CPU tensor
    res, info = srv.wait(t)             # BuildResult of views into the server's memory
    ...                                 # use res (valid until release)
    srv.release(t)

Requests queued while batches are on the GPU are coalesced into the next batched build; each
result is identical to BVHBuilder.build_soup of the request alone.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _native
from ._native import EBUSY, INPUT_HOST, OK, LvbhError


class _DeviceArray:
    """A raw device range exposed through __cuda_array_interface__ (zero-copy torch view)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def _view(ptr, shape, typestr, device):
    import torch
    if not ptr or 0 in shape:
        dt = {"<i4": torch.int32, "<f4": torch.float32}[typestr]
        return torch.empty(shape, dtype=dt, device=device)
    return torch.as_tensor(_DeviceArray(ptr, shape, typestr), device=device)


class Server:
    def __init__(self, device: int = 0, hbm_budget: int = 0, slots: int = 0,
                 max_batch_tris: int = 0, max_batch_reqs: int = 0, max_requests: int = 0):
        import torch
        self.device = torch.device("cuda", device)
        cfg = _native.ServerConfig(device=device, slots=slots, hbm_budget=hbm_budget,
                                   max_batch_tris=max_batch_tris, max_batch_reqs=max_batch_reqs,
                                   max_requests=max_requests)
        h = ctypes.c_void_p()
        rc = _native.lib.lvbh_server_create(ctypes.byref(h), ctypes.byref(cfg))
        if rc != OK:
            raise LvbhError(rc, "lvbh_server_create failed")
        self._h = h
        self._keep = {}  # ticket -> input kept alive until the request finishes

    def close(self):
        if getattr(self, "_h", None):
            # at interpreter exit the module's globals may already be gone
            lib = getattr(_native, "lib", None) if _native is not None else None
            if lib is not None:
                lib.lvbh_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        self.close()

    def _check(self, rc):
        if rc not in (OK, EBUSY):
            raise LvbhError(rc, _native.lib.lvbh_server_last_error(self._h).decode())

    def submit(self, tri, bounds=None) -> int:
        """tri: (N, 12) float32 CUDA tensor (device input), or host numpy array / CPU tensor
        (pinned memory lets its copy overlap the GPU work).  bounds: 6 floats or None."""
        import torch
        if isinstance(tri, torch.Tensor) and tri.is_cuda:
            tri = tri.contiguous().reshape(-1, 12)
            ptr, flags = tri.data_ptr(), 0
        else:
            if isinstance(tri, torch.Tensor):
                tri = tri.contiguous().reshape(-1, 12)
                ptr = tri.data_ptr()
            else:
                tri = np.ascontiguousarray(tri, dtype=np.float32).reshape(-1, 12)
                ptr = tri.ctypes.data
            flags = INPUT_HOST
        n = int(tri.shape[0])
        b = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float32).reshape(6)
        t = ctypes.c_uint64()
        rc = _native.lib.lvbh_submit(self._h, ctypes.c_void_p(ptr or None), n,
                                     None if b is None else b.ctypes.data_as(ctypes.c_void_p),
                                     flags, ctypes.byref(t))
        if rc != OK:
            raise LvbhError(rc, _native.lib.lvbh_server_last_error(self._h).decode())
        self._keep[t.value] = tri
        return t.value

    def _result(self, r: _native.Result):
        from . import BuildResult
        n, d = int(r.num_tris), self.device
        return BuildResult(nodes=_view(r.nodes, (n, 16), "<i4", d), tris=_view(r.tris, (n, 12), "<f4", d),
                           parents=_view(r.parents, (2 * n,), "<i4", d),
                           leaf_index=_view(r.leaf_index, (n,), "<i4", d),
                           morton=_view(r.morton, (n,), "<i4", d),
                           bounds=np.array(r.bounds[:], dtype=np.float32))

    @staticmethod
    def _info(i: _native.RequestInfo) -> dict:
        return {"status": i.status, "num_tris": i.num_tris, "batch_reqs": i.batch_reqs,
                "batch_tris": i.batch_tris, "queued_ms": i.queued_ms, "latency_ms": i.latency_ms}

    def poll(self, ticket: int):
        """(BuildResult, info) once finished, None while queued or running."""
        r, i = _native.Result(), _native.RequestInfo()
        rc = _native.lib.lvbh_poll(self._h, ticket, ctypes.byref(r), ctypes.byref(i))
        if rc == EBUSY:
            return None
        self._keep.pop(ticket, None)
        self._check(rc)
        return self._result(r), self._info(i)

    def wait(self, ticket: int, timeout_ms: int = -1):
        r, i = _native.Result(), _native.RequestInfo()
        rc = _native.lib.lvbh_wait(self._h, ticket, int(timeout_ms), ctypes.byref(r), ctypes.byref(i))
        if rc == EBUSY:
            return None
        self._keep.pop(ticket, None)
        self._check(rc)
        return self._result(r), self._info(i)

    def release(self, ticket: int):
        rc = _native.lib.lvbh_request_release(self._h, ticket)
        if rc != OK:
            raise LvbhError(rc, "lvbh_request_release")
        self._keep.pop(ticket, None)

    def stats(self) -> dict:
        s = _native.ServerStats()
        self._check(_native.lib.lvbh_server_stats_get(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_ if k != "pad"}
