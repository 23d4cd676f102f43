"""Every kernel launched with programmatic stream serialisation must wait for the kernel before
it (chain_wait) before it touches global memory; a chained kernel without the wait would read
its predecessor's output while that kernel still runs.  Checked on the sources (no GPU)."""
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "webgpu-lvbh-demo_b200", "csrc")


def _sources():
    out = {}
    for name in os.listdir(CSRC):
        if name.endswith((".cu", ".cuh", ".h")):
            with open(os.path.join(CSRC, name)) as f:
                out[name] = f.read()
    return out


def _kernel_body(text, kernel):
    m = re.search(r"__global__[^{;]*?\b" + kernel + r"\s*\(", text)
    if not m:
        return None
    i = text.index("{", m.end())
    depth = 0
    for j in range(i, len(text)):
        depth += {"{": 1, "}": -1}.get(text[j], 0)
        if depth == 0:
            return text[i:j + 1]
    raise AssertionError(f"unbalanced body of {kernel}")


def test_every_chained_kernel_waits_first():
    src = _sources()
    chained = set()
    for text in src.values():
        for m in re.finditer(r"launch_chained\(\s*[^,]+,\s*(k_\w+)", text):
            chained.add(m.group(1))
    assert {"k_morton_cen", "k_tile_hist", "k_chunk_scan", "k_scatter", "k_tree_climb",
            "k_top_group"} <= chained, chained
    for kernel in sorted(chained):
        bodies = [b for b in (_kernel_body(t, kernel) for t in src.values()) if b]
        assert len(bodies) == 1, kernel
        body = bodies[0]
        assert "chain_wait();" in body, kernel
        before = body[:body.index("chain_wait();")]
        # nothing before the wait may read or write global memory: only shared-memory set-up
        for pattern in (r"__ldg", r"ld_relaxed_gpu", r"\bctl->", r"\*epoch", r"atomic\w*\(",
                        r"\bkeys\w*\[", r"\bitems\[", r"\bcounts\[", r"\bcen\["):
            assert not re.search(pattern, before), (kernel, pattern)


def test_the_wait_is_griddepcontrol():
    text = _sources()["lvbh_device.cuh"]
    body = text[text.index("void chain_wait()"):]
    body = body[:body.index("}") + 1]
    assert "griddepcontrol.wait" in body
    assert "launch_dependents" not in body
