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
