"""Extract the golden arrays of elsa's blob / B-spline tests into tests/golden/voxel_luts.json.

Reads the reference test sources as text (C++ doctest files; nothing is compiled or run):
  elsa/projectors/tests/test_Luts.cpp            ProjectedBlobLut (a=2, alpha=10.83, m=2, 101
                                                 samples) and ProjectedBSplineLut (order 3, dim 2)
  elsa/projectors/tests/test_BlobDerivative.cpp  projected blob derivative, a=1, alpha in
                                                 {2.5, 5, 7.5, 10.83}, m in {1, 2}, s = i/100
  elsa/projectors/tests/test_BlobGradientHelper.cpp  the same arrays (used there as expected[i]/s)

Usage: python tests/golden/make_voxel_goldens.py <reference_root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def _numbers(text):
    return [float(v) for v in re.findall(NUM, text)]


def _brace_block(text, start):
    """Contents of the {...} block whose opening brace is at or after `start`."""
    i = text.index("{", start)
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i + 1:j], j
    raise ValueError("unbalanced braces")


def lut_goldens(src):
    out = {}
    for key, marker in (("projected_blob_lut_a2_alpha10.83_m2",
                         'TEST_CASE_TEMPLATE("ProjectedBlobLut: "'),
                        ("projected_bspline_lut_order3_dim2",
                         'TEST_CASE_TEMPLATE("ProjectedBSplineLut: "')):
        at = src.index(marker)
        body, _ = _brace_block(src, src.index("expected", at))
        vals = _numbers(body)
        assert len(vals) == 101, (key, len(vals))
        out[key] = vals
    return out


def derivative_goldens(src):
    """getExpected(a, alpha, m): nested if (a == .), if (alpha == .), if (m == .) + return {..}."""
    body, _ = _brace_block(src, src.index("getExpected(data_t a, data_t alpha, data_t m)\n"))
    out = {}
    a = alpha = m = None
    pos = 0
    pat = re.compile(r"if \((a|alpha|m) == (?:Approx\()?(" + NUM + r")\)?\)|return \{")
    while True:
        mt = pat.search(body, pos)
        if not mt:
            break
        if mt.group(1) == "a":
            a = float(mt.group(2))
            pos = mt.end()
        elif mt.group(1) == "alpha":
            alpha = float(mt.group(2))
            pos = mt.end()
        elif mt.group(1) == "m":
            m = int(float(mt.group(2)))
            pos = mt.end()
        else:
            block, end = _brace_block(body, mt.start())
            vals = _numbers(block)
            if a is not None and alpha is not None and m is not None and len(vals) == 101:
                out["a%g_alpha%g_m%d" % (a, alpha, m)] = vals
            pos = end + 1
            m = None  # the next return belongs to a new (alpha, m) branch
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: %s <root of the reference checkout>" % sys.argv[0])
    root = sys.argv[1]
    tests = os.path.join(root, "elsa", "projectors", "tests")
    with open(os.path.join(tests, "test_Luts.cpp")) as f:
        luts = lut_goldens(f.read())
    with open(os.path.join(tests, "test_BlobDerivative.cpp")) as f:
        deriv = derivative_goldens(f.read())
    with open(os.path.join(tests, "test_BlobGradientHelper.cpp")) as f:
        grad = derivative_goldens(f.read())
    assert grad == deriv  # stored once
    data = {
        "source": "elsa projectors/tests: test_Luts.cpp, test_BlobDerivative.cpp, "
                  "test_BlobGradientHelper.cpp (arrays copied as numbers)",
        "luts": luts,
        "blob_derivative_projected": deriv,
    }
    path = os.path.join(HERE, "voxel_luts.json")
    with open(path, "w") as f:
        json.dump(data, f, indent=0)
    print(path, {k: len(v) for k, v in data.items() if isinstance(v, dict)})


if __name__ == "__main__":
    main()
