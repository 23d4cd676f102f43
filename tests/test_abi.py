"""The C-ABI library: it loads, exports every entry point include/lvbh.h declares, the header
is plain C whose struct layout the ctypes binding matches, and argument errors come back as
status codes.  No GPU needed (nothing here launches a kernel)."""
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "lvbh.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"LVBH_API\s+[\w\s\*]*?\b(lvbh_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("lvbh_create", "lvbh_destroy", "lvbh_build_soup", "lvbh_build_indexed",
              "lvbh_sync", "lvbh_release", "lvbh_trace", "lvbh_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    import lvbh._native as nat
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT\s+(lvbh_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert hasattr(nat.lib, s)


def test_c_header_layout_and_host_errors(tmp_path):
    import lvbh._native as nat
    exe = tmp_path / "abi_check"
    libdir = os.path.dirname(nat.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "abi_check.c"), "-L", libdir, "-llvbh",
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    kv = dict(line.split(" ", 1) for line in out.strip().splitlines())
    import ctypes
    assert int(kv["sizeof_result"]) == ctypes.sizeof(nat.Result)
    assert int(kv["off_nodes"]) == nat.Result.nodes.offset
    assert int(kv["off_bounds"]) == nat.Result.bounds.offset
    assert int(kv["off_owned"]) == nat.Result.owned.offset
    assert int(kv["sizeof_config"]) == ctypes.sizeof(nat.Config)
    assert "sm_100a" in kv["version"]
    assert int(kv["sizeof_server_config"]) == ctypes.sizeof(nat.ServerConfig)
    assert int(kv["sizeof_tunables"]) == ctypes.sizeof(nat.Tunables) == 16
    assert int(kv["sizeof_request_info"]) == ctypes.sizeof(nat.RequestInfo)
    assert int(kv["off_latency"]) == nat.RequestInfo.latency_ms.offset
    assert int(kv["sizeof_server_stats"]) == ctypes.sizeof(nat.ServerStats)
    assert int(kv["off_max_batch_seen"]) == nat.ServerStats.max_batch_seen.offset
    assert int(kv["sizeof_pt_frame"]) == ctypes.sizeof(nat.PtFrame) == 32
    for k in ("build_null_ctx", "indexed_null_ctx", "sync_null", "release_null", "create_null",
              "stage_null", "trace_null", "copy_null", "batched_null_ctx", "server_create_null",
              "submit_null", "poll_null", "wait_null", "release_req_null", "stats_null",
              "set_tunables_null", "get_tunables_null", "parse_obj_null_ctx", "pt_null_ctx", "mesh_null_ctx",
              "trace_mesh_null_ctx"):
        assert int(kv[k]) == nat.EINVAL, k
    assert kv["server_error_null"] == "no server"
    assert kv["last_error_null"] == "no context"
    assert int(kv["scratch_1M"]) >= 12 * (1 << 20)


def test_no_cpu_fallback(monkeypatch, tmp_path):
    """Importing the binding without the compiled library fails loudly."""
    import importlib.util
    import lvbh._native as nat
    spec = importlib.util.spec_from_file_location("lvbh_native_probe", nat.__file__)
    mod = importlib.util.module_from_spec(spec)
    monkeypatch.setattr(os.path, "exists", lambda p: False if p.endswith("liblvbh.so") else os.path.isfile(p) or os.path.isdir(p))
    with pytest.raises(ImportError):
        spec.loader.exec_module(mod)


def test_create_without_gpu_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ctypes
    import lvbh._native as nat
    ctx = ctypes.c_void_p()
    rc = nat.lib.lvbh_create(ctypes.byref(ctx), None)
    assert rc != nat.OK and not ctx.value
