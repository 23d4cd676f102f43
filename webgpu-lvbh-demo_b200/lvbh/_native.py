"""ctypes binding of the C ABI declared in include/lvbh.h (liblvbh.so, built in-tree).

There is no fallback: when the compiled library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblvbh.so")

# status codes (include/lvbh.h)
OK, EINVAL, ENOMEM, ETIMEOUT, ECUDA, EBUSY, EDEVICE, ERANGE, EPARSE = 0, 1, 2, 3, 4, 5, 6, 7, 8
STATUS_NAMES = {OK: "LVBH_OK", EINVAL: "LVBH_EINVAL", ENOMEM: "LVBH_ENOMEM",
                ETIMEOUT: "LVBH_ETIMEOUT", ECUDA: "LVBH_ECUDA", EBUSY: "LVBH_EBUSY",
                EDEVICE: "LVBH_EDEVICE", ERANGE: "LVBH_ERANGE",
                EPARSE: "LVBH_EPARSE"}
NOALLOC_MAX_KEYS = 1 << 20

# build flags
INPUT_HOST, ASYNC, OUT_CALLER, PROFILE, NO_GRAPH, AUTOTUNE = 0x1, 0x2, 0x4, 0x8, 0x10, 0x20
MAX_TRIS = 1 << 29
NUM_STAGES = 7
STAGE_NAMES = ("upload", "bounds", "morton", "sort", "gather", "tree", "top")


class LvbhError(RuntimeError):
    """A non-zero status returned through the C ABI."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


class PtFrame(ctypes.Structure):
    """lvbh_pt_frame: the path tracer's uniform buffer (pos, rst, lat)."""
    _fields_ = [("pos", ctypes.c_float * 3), ("rst", ctypes.c_float), ("lat", ctypes.c_float * 3),
                ("pad", ctypes.c_float)]


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("reserve_tris", ctypes.c_uint32),
                ("reserved", ctypes.c_uint64 * 4)]


class Result(ctypes.Structure):
    _fields_ = [("num_tris", ctypes.c_uint32), ("num_nodes", ctypes.c_uint32),
                ("nodes", ctypes.c_void_p), ("tris", ctypes.c_void_p),
                ("parents", ctypes.c_void_p), ("leaf_index", ctypes.c_void_p),
                ("morton", ctypes.c_void_p), ("bounds", ctypes.c_float * 6),
                ("owned", ctypes.c_uint32)]


class Tunables(ctypes.Structure):
    _fields_ = [("digit_bits", ctypes.c_uint32), ("tree_block", ctypes.c_uint32),
                ("tree_ctas_per_sm", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_uint32),
                ("hbm_budget", ctypes.c_uint64), ("max_batch_tris", ctypes.c_uint32),
                ("max_batch_reqs", ctypes.c_uint32), ("max_requests", ctypes.c_uint32),
                ("pad", ctypes.c_uint32), ("reserved", ctypes.c_uint64 * 4)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("num_tris", ctypes.c_uint32),
                ("batch_reqs", ctypes.c_uint32), ("batch_tris", ctypes.c_uint32),
                ("queued_ms", ctypes.c_double), ("latency_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in
                ("submitted", "completed", "failed", "batches", "tris_built", "budget_bytes",
                 "result_bytes", "bytes_in_use", "peak_bytes", "admission_waits")] + \
               [("max_batch_seen", ctypes.c_uint32), ("pad", ctypes.c_uint32)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {os.path.dirname(HERE)}` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    vp, u32, i32 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int
    L.lvbh_version.restype = ctypes.c_char_p
    L.lvbh_version.argtypes = []
    L.lvbh_create.restype = i32
    L.lvbh_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(Config)]
    L.lvbh_destroy.restype = None
    L.lvbh_destroy.argtypes = [vp]
    L.lvbh_build_soup.restype = i32
    L.lvbh_build_soup.argtypes = [vp, vp, u32, vp, u32, ctypes.POINTER(Result), vp]
    L.lvbh_build_indexed.restype = i32
    L.lvbh_build_indexed.argtypes = [vp, vp, u32, vp, u32, vp, u32, ctypes.POINTER(Result), vp]
    L.lvbh_build_mesh.restype = i32
    L.lvbh_build_mesh.argtypes = [vp, vp, u32, vp, u32, vp, u32, ctypes.POINTER(Result), vp]
    L.lvbh_trace_mesh.restype = i32
    L.lvbh_trace_mesh.argtypes = [vp, vp, vp, vp, u32, u32, vp, u32, vp, vp, vp, vp]
    L.lvbh_build_batched.restype = i32
    L.lvbh_build_batched.argtypes = [vp, vp, vp, u32, vp, vp, u32, ctypes.POINTER(Result), vp]
    L.lvbh_set_tunables.restype = i32
    L.lvbh_set_tunables.argtypes = [vp, ctypes.POINTER(Tunables)]
    L.lvbh_get_tunables.restype = i32
    L.lvbh_get_tunables.argtypes = [vp, ctypes.POINTER(Tunables), ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_uint32)]
    L.lvbh_sync.restype = i32
    L.lvbh_sync.argtypes = [vp]
    L.lvbh_release.restype = i32
    L.lvbh_release.argtypes = [vp, ctypes.POINTER(Result)]
    L.lvbh_stage_times.restype = i32
    L.lvbh_stage_times.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.lvbh_scratch_bytes.restype = ctypes.c_size_t
    L.lvbh_scratch_bytes.argtypes = [u32]
    L.lvbh_last_error.restype = ctypes.c_char_p
    L.lvbh_last_error.argtypes = [vp]
    L.lvbh_copy_to_host.restype = i32
    L.lvbh_copy_to_host.argtypes = [vp, vp, vp, ctypes.c_size_t, vp]
    L.lvbh_sort_pairs_noalloc.restype = i32
    L.lvbh_sort_pairs_noalloc.argtypes = [vp, u32, vp, vp, vp]
    L.lvbh_test_stall_lookback.restype = i32
    L.lvbh_test_stall_lookback.argtypes = [vp, u32, u32]
    L.lvbh_server_create.restype = i32
    L.lvbh_server_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ServerConfig)]
    L.lvbh_server_destroy.restype = None
    L.lvbh_server_destroy.argtypes = [vp]
    L.lvbh_submit.restype = i32
    L.lvbh_submit.argtypes = [vp, vp, u32, vp, u32, ctypes.POINTER(ctypes.c_uint64)]
    L.lvbh_poll.restype = i32
    L.lvbh_poll.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(Result), ctypes.POINTER(RequestInfo)]
    L.lvbh_wait.restype = i32
    L.lvbh_wait.argtypes = [vp, ctypes.c_uint64, i32, ctypes.POINTER(Result), ctypes.POINTER(RequestInfo)]
    L.lvbh_request_release.restype = i32
    L.lvbh_request_release.argtypes = [vp, ctypes.c_uint64]
    L.lvbh_server_stats_get.restype = i32
    L.lvbh_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.lvbh_server_last_error.restype = ctypes.c_char_p
    L.lvbh_server_last_error.argtypes = [vp]
    L.lvbh_trace.restype = i32
    L.lvbh_trace.argtypes = [vp, vp, vp, u32, vp, u32, vp, vp, vp, vp]
    L.lvbh_pt_sample.restype = i32
    L.lvbh_pt_sample.argtypes = [vp, vp, vp, u32, vp, vp, u32, u32, ctypes.POINTER(PtFrame), vp]
    L.lvbh_parse_obj.restype = i32
    L.lvbh_parse_obj.argtypes = [vp, vp, ctypes.c_uint64, u32, ctypes.POINTER(vp), ctypes.POINTER(u32),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64), vp]
    return L


lib = _load()


def version() -> str:
    return lib.lvbh_version().decode()


def check(ctx, rc: int):
    if rc != OK:
        msg = lib.lvbh_last_error(ctx).decode() if ctx else "no context"
        raise LvbhError(rc, msg)
