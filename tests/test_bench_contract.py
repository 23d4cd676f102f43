"""The benchmark's fixed tables agree with the committed profile summaries (CPU only).

bench.py reports, besides its measured times, figures it takes from tables: the traffic model
(340 bytes per triangle), the DRAM bytes of the dominant kernel (profiles/traffic.json, from an
ncu capture) and the number of kernels it launches per build.  These tests keep the tables and
the committed summaries from drifting apart.
"""
import json
import os
import re

import bench

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_traffic_model_total():
    assert bench.MODEL_TOTAL == 340
    assert sum(bench.MODEL_BYTES.values()) == bench.MODEL_TOTAL


def test_every_timed_kernel_has_captured_traffic():
    with open(os.path.join(REPO, "profiles", "traffic.json")) as f:
        kernels = json.load(f)["kernels"]
    for stage, (name, launches) in bench.KERNELS.items():
        if name is None:
            continue
        assert name in kernels, (stage, name)
        assert kernels[name]["dram_bytes_per_tri"] > 0
        assert launches >= 1
    # the dominant kernel's traffic scales with the triangle count
    n = 1 << 24
    t = bench.load_traffic("k_tree_climb", n)
    assert t == kernels["k_tree_climb"]["dram_bytes_per_tri"] * n
    # and stays above its algorithmic bytes (gather lines are fetched whole)
    assert t > bench.MODEL_BYTES["tree"] * n


def test_launches_per_build_match_the_launch_list():
    """The committed launch list of the 16.7 M build: 15 builds, LAUNCHES_PER_BUILD each."""
    with open(os.path.join(REPO, "profiles", "launches_clustered16M.md")) as f:
        text = f.read()
    builds = int(re.search(r"\((\d+) builds;", text).group(1))
    rows = re.findall(r"^\| (k_\w+) \| (\d+) \|", text, flags=re.M)
    total = sum(int(c) for _, c in rows)
    assert total == builds * bench.LAUNCHES_PER_BUILD, (total, builds)
    per_kernel = {k: int(c) // builds for k, c in rows}
    for stage, (name, launches) in bench.KERNELS.items():
        if name is not None:
            assert per_kernel[name] == (1 if stage == "top" else launches), (stage, name)


def test_reference_arm_loads_no_project_cuda_library():
    """bench.py --impl reference runs the oracle only: in a fresh process, after a run of the
    arm on the 65,536-triangle workload, neither the lvbh package nor liblvbh.so is loaded,
    and the line names the full workload it timed."""
    import json
    import subprocess
    import sys
    code = (
        "import io, json, sys, contextlib\n"
        "sys.path.insert(0, %r)\n"
        "import bench\n"
        "class A: workload, warmup, steps = 'uniform64K', 1, 1\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf): bench.run_reference(A, 1, 0)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'line': json.loads(buf.getvalue()), 'lvbh_loaded': 'liblvbh.so' in maps,\n"
        "                  'lvbh_imported': 'lvbh' in sys.modules}))\n" % REPO)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, check=True)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    assert not r["lvbh_loaded"] and not r["lvbh_imported"]
    line = r["line"]
    assert line["impl"] == "reference" and line["config"]["num_tris"] == 65_536
    assert "one full build" in line["cpu_baseline"]["sample"]
