"""The OBJ ingest oracle (oracle/obj_oracle.cpp) against hand-derived known answers.

No JavaScript engine runs here, so the expected soups and bounds in obj_cases.CASES are worked
out from scripts/obj/obj-file-parser.js and scripts/obj/parse-obj.js by hand: fan order, the y/z
swap, model-0 selection, negative and hexadecimal indices, parseFloat prefixes, Math.min /
Math.max with NaN and signed zeros, float32 rounding, JavaScript whitespace, and every statement
the reference's parser throws on.
"""
import numpy as np
import pytest

import oracle
from obj_cases import CASES, same_f32, same_f64, soup_rows, messy_obj


@pytest.mark.parametrize("name,text,expected", CASES, ids=[c[0] for c in CASES])
def test_oracle_known_answers(name, text, expected):
    if expected[0] == "throws":
        with pytest.raises(oracle.ObjThrows) as e:
            oracle.parse_obj(text)
        assert e.value.line == expected[1]
        return
    _, rows, bounds = expected
    tri, b = oracle.parse_obj(text)
    assert same_f64(b, np.array(bounds, dtype=np.float64)), (b, bounds)
    assert same_f32(tri, soup_rows(rows, b)), (tri, soup_rows(rows, b))


def test_oracle_messy_texts_parse():
    """The generated texts the GPU tests use parse without a throw, to a soup with the floor."""
    for seed in range(4):
        tri, b = oracle.parse_obj(messy_obj(seed, lines=500))
        assert tri.shape[0] >= 2 and tri.shape[1] == 12
        assert np.all(tri[:, 3] == np.float32(3.1415))
