"""OBJ ingest on the GPU (lvbh_parse_obj, through the C ABI) against the oracle, bit for bit.

The soup (every float32 word, NaN as one value) and the six BOUNDS doubles must equal the
oracle's; where the oracle throws, the device parse must fail with LVBH_EPARSE at the same line.
Text comes from host memory, from device memory, and from device memory at an odd address.
"""
import math
from decimal import Decimal, getcontext
from fractions import Fraction

import numpy as np
import pytest

import oracle
from obj_cases import CASES, messy_obj, same_f32, same_f64

pytestmark = pytest.mark.gpu


def gpu_parse(builder, text: bytes, where="host"):
    import torch
    if where == "host":
        out = builder.parse_obj(text)
    else:
        off = 1 if where == "device_odd" else 0
        buf = torch.zeros(len(text) + off, dtype=torch.uint8)
        if text:
            buf[off:] = torch.frombuffer(bytearray(text), dtype=torch.uint8)
        out = builder.parse_obj(buf.cuda()[off:])
    return out["TRI_ARR"].cpu().numpy(), np.array(out["BOUNDS"]["min"] + out["BOUNDS"]["max"])


def check_same(builder, text, where="host", tag=""):
    import lvbh
    if isinstance(text, str):
        text = text.encode("utf-8")
    try:
        ref_tri, ref_b = oracle.parse_obj(text)
        ref_line = None
    except oracle.ObjThrows as e:
        ref_line = e.line
    if ref_line is not None:
        with pytest.raises(lvbh.ObjError) as e:
            gpu_parse(builder, text, where)
        assert e.value.line == ref_line, f"{tag}: line {e.value.line} vs {ref_line}"
        return None
    tri, b = gpu_parse(builder, text, where)
    assert same_f64(b, ref_b), f"{tag}: bounds {b} vs {ref_b}"
    assert tri.shape == ref_tri.shape, f"{tag}: {tri.shape} vs {ref_tri.shape}"
    if not same_f32(tri, ref_tri):
        bad = np.nonzero(~((tri.view(np.uint32) == ref_tri.view(np.uint32)) |
                           (np.isnan(tri) & np.isnan(ref_tri))))
        raise AssertionError(f"{tag}: {bad[0].size} words differ, first rows {np.unique(bad[0])[:8]}")
    return tri, b


@pytest.mark.parametrize("where", ["host", "device", "device_odd"])
def test_known_cases(builder, where):
    for name, text, _ in CASES:
        check_same(builder, text, where, name)


@pytest.mark.parametrize("seed", range(6))
def test_messy_texts(builder, seed):
    lines = [300, 3000, 30000, 120000, 4000, 50000][seed]
    text = messy_obj(seed, lines=lines, objects=1 + seed % 3)
    for where in ("host", "device_odd"):
        check_same(builder, text, where, f"seed {seed} {where}")


def number_strings(seed=7, count=2400):
    """Decimal literals across the device's paths: short (one IEEE operation), long
    significands (exact 128-bit path), past 19 digits, exponents past +-27 (host path), exact
    halfway points between doubles and their neighbours, and the edges of the double range."""
    rng = np.random.default_rng(seed)
    out = ["9007199254740993", "9007199254740995", "18446744073709551615", "18446744073709551616",
           "18446744073709551617", "1e23", "8.98846567431158e307", "1.7976931348623157e308",
           "1.7976931348623159e308", "2.2250738585072014e-308", "2.2250738585072011e-308",
           "4.9406564584124654e-324", "2.4703282292062327e-324", "2.4703282292062328e-324",
           "1e-400", "1e400", "0.000000000000000000000000000001", "123456789012345678901234567890",
           "1e27", "1e28", "1e-27", "1e-28", "7.450580596923828125e-9", "0.1", "0.3", "-0.0"]
    for _ in range(count // 3):
        nd = int(rng.integers(1, 26))
        d = "".join(str(int(c)) for c in rng.integers(0, 10, nd))
        p = int(rng.integers(0, nd + 1))
        s = d[:p] + "." + d[p:] if p < nd else d
        e = int(rng.integers(-35, 36))
        out.append(("-" if rng.random() < 0.3 else "") + s + (f"e{e}" if rng.random() < 0.6 else ""))
    getcontext().prec = 1200
    for _ in range(count // 3):
        x = float(rng.normal() * 10.0 ** int(rng.integers(-25, 26)))
        y = math.nextafter(x, math.inf)
        mid = (Fraction(x) + Fraction(y)) / 2
        exact = Decimal(mid.numerator) / Decimal(mid.denominator)
        t = format(exact, "f")
        k = int(rng.integers(3))
        if k == 1:
            t = t + "000000001"  # just above the tie
        elif k == 2 and len(t.replace("-", "").replace(".", "").lstrip("0")) > 20:
            t = t[:-1]  # just below the tie
        out.append(t)
    for _ in range(count - len(out)):
        x = float(rng.normal() * 10.0 ** int(rng.integers(-30, 31)))
        out.append(["%.17g", "%.16g", "%.15g", "%.9g", "%.6f", "%.20e"][int(rng.integers(6))] % x)
    return out


def test_parse_float_exact(builder):
    """Every literal parses to the correctly rounded double (the bounds carry it unrounded):
    the oracle's strtod, Python's float() and the device agree."""
    nums = number_strings()
    for i in range(0, len(nums) - 2, 3):
        a, b, c = nums[i:i + 3]
        text = f"v {a} {b} {c}\nv {a} {b} {c}\nv {a} {b} {c}\nf 1 2 3\n"
        got = check_same(builder, text, "host", f"numbers {a} {b} {c}")
        v = np.array([float(a), float(c), float(b)])
        # BOUNDS start at +-1e30 (parse-obj.js:10-16): the value shows in min, max or both
        want = np.concatenate([np.where(v < 1e30, v, 1e30), np.where(v > -1e30, v, -1e30)])
        want[np.concatenate([np.isnan(v), np.isnan(v)])] = np.nan
        _, bounds = got
        assert same_f64(bounds, want), (a, b, c, bounds, want)


def test_sphere_obj_then_build(builder):
    """OBJ text of a 525k-triangle mesh -> device soup -> build, against oracle parse -> oracle
    build: main.js's path (parseObj, then build(TRI_ARR, NUM_TRIS, BOUNDS))."""
    from lvbh import scenes
    from test_parity_gpu import assert_same
    xyz, idx = scenes.sphere_mesh(512, seed=3, indexed=True)
    text = scenes.obj_text(xyz, idx)
    tri, b = check_same(builder, text, "host", "sphere")
    out = builder.parse_obj(text)
    bounds32 = np.array(out["BOUNDS"]["min"] + out["BOUNDS"]["max"], dtype=np.float32)
    res = builder.build_soup(out["TRI_ARR"], bounds32).to_numpy()
    ref = oracle.build(tri, bounds32, threads=0)
    assert_same(res, ref, "sphere build")


def test_reuse_and_growth(builder):
    """Parses of growing and shrinking texts on one context reuse and grow its buffers; each
    result is complete and right."""
    for seed, lines in ((10, 100), (11, 40000), (12, 50), (13, 80000)):
        check_same(builder, messy_obj(seed, lines=lines), "host", f"seed {seed}")


def test_lines_longer_than_the_window(builder):
    """Lines past a block's 24 KB shared-memory window are read from global memory by the same
    scanners: a face of 12,000 vertices, a vertex line padded with 100 KB of whitespace and a
    comment, and ordinary lines around them in the same blocks."""
    rng = np.random.default_rng(3)
    nv = 12_000
    lines = ["o big"]
    lines += ["v %.6f %.6f %.6f" % tuple(rng.normal(size=3)) for _ in range(nv)]
    lines.insert(5, "v 1.5" + " " * 100_000 + "2.5\t3.5 # " + "c" * 30_000)
    lines.append("f " + " ".join(str(i + 1) for i in range(nv)))
    lines.append("f " + " ".join("-%d/1/1" % (k + 1) for k in range(3)))
    lines.append("f 1 2 3 " + " " * 9000 + "4")
    text = "\n".join(lines) + "\n"
    for where in ("host", "device"):
        check_same(builder, text, where, f"long lines {where}")
    with_throw = text + "g" + " " * 50_000 + "\n"
    check_same(builder, with_throw, "host", "long throwing line")
