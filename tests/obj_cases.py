"""OBJ ingest test cases: texts with the results the reference's parseObj gives for them.

Each case is (name, text, expected).  `expected` is ("throws", line) where the reference throws
(line: the 1-based line of the rejected statement, 0 for a failure after parsing), or
("soup", rows, bounds): the model's triangles as (x, y, z) vertex triples after the y/z swap
(the floor and the pad are added by `soup_rows`), and the six BOUNDS doubles.  The expected
values follow scripts/obj/obj-file-parser.js:19-193 and scripts/obj/parse-obj.js:3-88 by hand:
they pin the oracle, and the GPU tests compare the device ingest with the oracle on the same
texts.
"""
import numpy as np

PAD = np.float32(3.1415)
INF = float("inf")
NAN = float("nan")

QUAD = "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 2\n"

CASES = [
    # fan triangulation from the first vertex, y and z swapped (parse-obj.js:17-60)
    ("quad_fan", QUAD + "f 1 2 3 4\n",
     ("soup", [[(0, 0, 0), (1, 0, 0), (1, 0, 1)], [(0, 0, 0), (1, 0, 1), (0, 2, 1)]],
      [0, 0, 0, 1, 2, 1])),
    ("slashes", QUAD + "vt 0 0\nvn 0 0 1\nf 1/1/1 2/1/1 3//1\n",
     ("soup", [[(0, 0, 0), (1, 0, 0), (1, 0, 1)]], [0, 0, 0, 1, 0, 1])),
    # negative indices count back from the vertices defined so far (obj-file-parser.js:180)
    ("negative", "v 0 0 0\nv 1 0 0\nv 2 0 0\nf -1 -2 -3\nv 5 5 5\n",
     ("soup", [[(2, 0, 0), (1, 0, 0), (0, 0, 0)]], [0, 0, 0, 2, 0, 0])),
    ("hex_index", "v 0 0 0\nv 1 0 0\nv 0 0 1\nf 0x1 0X2 3\n",
     ("soup", [[(0, 0, 0), (1, 0, 0), (0, 1, 0)]], [0, 0, 0, 1, 1, 0])),
    ("index_prefix", "v 0 0 0\nv 1 0 0\nv 0 0 1\nf 1abc 2.9 3e5\n",
     ("soup", [[(0, 0, 0), (1, 0, 0), (0, 1, 0)]], [0, 0, 0, 1, 1, 0])),
    # model 0: the default model when geometry precedes the first `o` ...
    ("default_model_first", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\no a\nv 7 7 7\nv 7 7 7\nv 7 7 7\nf 1 2 3\n",
     ("soup", [[(0, 0, 0), (1, 0, 0), (0, 0, 1)]], [0, 0, 0, 1, 0, 1])),
    # ... else the model the first `o` opens; g and s create no model
    ("first_object", "g grp\ns 1\no a\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\no b\nv 9 9 9\nv 9 9 9\nv 9 9 9\nf 1 2 3\n",
     ("soup", [[(0, 0, 0), (1, 0, 0), (0, 0, 1)]], [0, 0, 0, 1, 0, 1])),
    ("empty_first_object", "o a\no b\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
     ("soup", [], [1e30, 1e30, 1e30, -1e30, -1e30, -1e30])),
    ("line_creates_model", "l 1 2\n", ("soup", [], [1e30, 1e30, 1e30, -1e30, -1e30, -1e30])),
    ("vt_creates_model", "vt 0 0\n", ("soup", [], [1e30, 1e30, 1e30, -1e30, -1e30, -1e30])),
    # tokenising: '#' comments, runs of whitespace, CRLF, keyword case, JavaScript \s
    ("crlf_tabs_case", "  V\t1\t2\t3 \r\nv 4 5 6\r\n\r\nv 7 8 9 # comment\r\nF 1 2 3\r\n",
     ("soup", [[(1, 3, 2), (4, 6, 5), (7, 9, 8)]], [1, 3, 2, 7, 9, 8])),
    ("comment_cuts", "v 1 2 #3\nv 4#5 6\nv 7 8 9\nf 1 2 3 # 4\n",
     ("soup", [[(1, 0, 2), (4, 0, 0), (7, 9, 8)]], [1, 0, 0, 7, 9, 8])),
    ("unicode_spaces", "\ufeffv\u00a01\u20002\u30003\nv\u20284 5 6\nv 7\u202f8\ufeff9\nf\u00a01 2 3\u2029\n",
     ("soup", [[(1, 3, 2), (4, 6, 5), (7, 9, 8)]], [1, 3, 2, 7, 9, 8])),
    ("non_space_unicode", "v 1\u00e92 3 4\nv\u00e9 9 9 9\nv 0 0 0\nv 1 1 1\nf 1 2 3\n",
     ("soup", [[(1, 4, 3), (0, 0, 0), (1, 1, 1)]], [0, 0, 0, 1, 4, 3])),
    # parseFloat: longest decimal prefix, Infinity, NaN, missing coordinates are 0
    ("parse_float_forms", "v 1e 2.5e+ -.5\nv +3 0x10 7.\nv 1.5E2 -2e-1 5\nf 1 2 3\n",
     ("soup", [[(1, -0.5, 2.5), (3, 7, 0), (150, 5, -0.2)]], [1, -0.5, -0.2, 150, 7, 2.5])),
    ("missing_coords", "v 1\nv 2 3\nv\nf 1 2 3\n",
     ("soup", [[(1, 0, 0), (2, 0, 3), (0, 0, 0)]], [0, 0, 0, 2, 0, 3])),
    ("infinity", "v Infinity -Infinity 1\nv 0 0 0\nv 0 0 0\nf 1 2 3\n",
     ("soup", [[(INF, 1, -INF), (0, 0, 0), (0, 0, 0)]], [0, 0, -INF, INF, 1, 0])),
    ("nan_absorbs", "v . 1 1\nv 2 2 2\nv 3 3 3\nf 1 2 3\n",
     ("soup", [[(NAN, 1, 1), (2, 2, 2), (3, 3, 3)]], [NAN, 1, 1, NAN, 3, 3])),
    ("signed_zero", "v -0 0 -0\nv 0 -0 0\nv 0 0 0\nf 1 2 3\n",
     ("soup", [[(-0.0, -0.0, 0), (0, 0, -0.0), (0, 0, 0)]], [-0.0, -0.0, -0.0, 0, 0, 0])),
    # float32 rounding of the doubles (Float32Array, build-bvh.js:14-21)
    ("f32_rounding", "v 0.1 16777217 16777219\nv 9007199254740993 1e-50 3.4028235677973366e38\nv 0 0 0\nf 1 2 3\n",
     ("soup", [[(0.1, 16777219, 16777217), (9007199254740992.0, 3.4028235677973366e38, 1e-50), (0, 0, 0)]],
      [0, 0, 0, 9007199254740992.0, 3.4028235677973366e38, 16777217])),
    # statements the parser rejects (the line of the first one)
    ("g_no_arg", "v 0 0 0\ng\n", ("throws", 2)),
    ("g_two_args", "v 0 0 0\ng a b\n", ("throws", 2)),
    ("s_no_arg", "s\n", ("throws", 1)),
    ("l_one_vertex", "v 0 0 0\nl 1\n", ("throws", 2)),
    ("l_three_parts", "v 0 0 0\nl 1/2/3 1\n", ("throws", 2)),
    ("f_two_vertices", QUAD + "f 1 2\n", ("throws", 5)),
    ("f_zero_index", QUAD + "f 1 0 2\n", ("throws", 5)),
    ("f_minus_zero", QUAD + "f -0 1 2\n", ("throws", 5)),
    ("f_hex_zero", QUAD + "f 0x0 1 2\n", ("throws", 5)),
    ("f_four_parts", QUAD + "f 1/1/1/1 2 3\n", ("throws", 5)),
    ("first_error_wins", "v 0 0 0\ng\nf 1 2\n", ("throws", 2)),
    ("error_in_other_model", QUAD + "f 1 2 3\no b\nf 1 2\n", ("throws", 7)),
    # failures after parsing: no model, a face naming no vertex of model 0
    ("empty_text", "", ("throws", 0)),
    ("only_comments", "# nothing\n\n   \n", ("throws", 0)),
    ("group_only", "g a\n", ("throws", 0)),
    ("index_out_of_range", "v 0 0 0\nv 0 0 0\nv 0 0 0\nf 1 2 4\n", ("throws", 0)),
    ("index_nan", QUAD + "f a b c\n", ("throws", 0)),
    ("negative_too_far", "v 0 0 0\nv 0 0 0\nf -1 -2 -3\n", ("throws", 0)),
    ("index_in_later_model_only", "v 0 0 0\no b\nv 1 1 1\nv 1 1 1\nv 1 1 1\no c\n"
     "v 0 0 0\nf 1 2 3\n", ("soup", [], [1e30, 1e30, 1e30, -1e30, -1e30, -1e30])),
    ("face_beyond_model0", "v 0 0 0\nv 0 0 0\nf 1 2 3\no b\nv 1 1 1\n", ("throws", 0)),
]


def soup_rows(rows, bounds):
    """Expected (N + 2, 12) float32 soup: the model's triangles and the two floor triangles
    at z_min + .01 (parse-obj.js:62-76), pad 3.1415."""
    out = []
    with np.errstate(over="ignore"):  # values past the float32 range round to infinity
        for t in rows:
            r = []
            for v in t:
                r += [np.float32(v[0]), np.float32(v[1]), np.float32(v[2]), PAD]
            out.append(r)
    h = np.float32(np.float64(bounds[2]) + 0.01)
    s = np.float32(10000.0)
    out.append([-s, -s, h, PAD, s, -s, h, PAD, -s, s, h, PAD])
    out.append([s, -s, h, PAD, s, s, h, PAD, -s, s, h, PAD])
    return np.array(out, dtype=np.float32).reshape(-1, 12)


def same_f32(a, b):
    """Bitwise equality of float32 arrays, every NaN as one value."""
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a.view(np.uint32)[~na], b.view(np.uint32)[~nb]))


def same_f64(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    na, nb = np.isnan(a), np.isnan(b)
    return bool(np.array_equal(na, nb) and np.array_equal(a.view(np.uint64)[~na], b.view(np.uint64)[~nb]))


def messy_obj(seed: int, lines: int = 2000, objects: int = 3) -> bytes:
    """A seeded OBJ text in many exporters' styles at once: several objects (model 0 first or
    after a default model), v lines with 1-4 numbers in decimal, exponent, signed, padded and
    long (17-25 digit) forms, vt / vn / s / g / l / usemtl lines, faces of 3-7 vertices with
    positive, negative and v/vt/vn indices, comments, CRLF and tab / Unicode whitespace."""
    rng = np.random.default_rng(seed)
    spaces = [" ", "  ", "\t", " \t", "\u00a0", "\u2003"]

    def sp():
        return spaces[rng.integers(len(spaces))] if rng.random() < 0.2 else " "

    def num():
        k = rng.integers(10)
        x = rng.normal() * 10.0 ** rng.integers(-3, 4)
        if k < 4:
            return "%.6f" % x
        if k == 4:
            return "%.17g" % x
        if k == 5:
            return "%.3e" % x
        if k == 6:
            return "%+.4f" % x
        if k == 7:
            return repr(float(np.float32(x)))
        if k == 8:  # long significands: past 19 digits, and halfway-like tails
            d = "".join(str(int(c)) for c in rng.integers(0, 10, rng.integers(18, 26)))
            return ("-" if rng.random() < 0.5 else "") + d[:3] + "." + d[3:]
        return "%d" % int(x * 100)

    out = []
    nobj_started = 0
    counts = [0]  # vertices of the current model
    default_first = rng.random() < 0.5
    if not default_first:
        out.append("o obj0")
        nobj_started = 1
    for i in range(lines):
        r = rng.random()
        nv = counts[-1]
        if r < 0.45 or nv < 3:
            k = rng.integers(1, 5)
            out.append("v" + "".join(sp() + num() for _ in range(k)))
            counts[-1] += 1
        elif r < 0.8:
            k = int(rng.integers(3, 8))
            toks = []
            for _ in range(k):
                j = int(rng.integers(1, nv + 1))
                if rng.random() < 0.3:
                    j = j - nv - 1  # negative form of the same vertex
                form = rng.integers(4)
                toks.append(str(j) if form == 0 else f"{j}/{j}" if form == 1 else f"{j}//{j}" if form == 2
                            else f"{j}/{j}/{j}")
            out.append(("f" if rng.random() < 0.9 else "F") + "".join(sp() + t for t in toks))
        elif r < 0.86:
            out.append("vn %s %s %s" % (num(), num(), num()))
        elif r < 0.9:
            out.append("vt %s %s" % (num(), num()))
        elif r < 0.93:
            out.append("# comment %d f 1 2" % i)
        elif r < 0.95:
            out.append("s %s" % ("off" if rng.random() < 0.5 else "1"))
        elif r < 0.96:
            out.append("g group%d" % i)
        elif r < 0.97:
            out.append("usemtl m%d" % i)
        elif r < 0.975:
            out.append("l 1 2")
        elif r < 0.98 and nobj_started < objects:
            out.append("o obj%d" % nobj_started)
            nobj_started += 1
            counts.append(0)
        else:
            out.append("v %s %s %s # trailing" % (num(), num(), num()))
            counts[-1] += 1
    eol = "\r\n" if rng.random() < 0.3 else "\n"
    return (eol.join(out) + eol).encode("utf-8")
