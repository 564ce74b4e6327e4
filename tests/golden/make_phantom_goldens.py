"""Extract the 16 x 16 modified Shepp-Logan golden array of elsa's phantom test into
tests/golden/shepp_logan_2d_16.json.

Reads elsa/generators/tests/test_Phantoms.cpp:145-187 as text (the `expected` vector, x fastest).
Usage: python tests/golden/make_phantom_goldens.py <reference_root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: %s <root of the reference checkout>" % sys.argv[0])
    root = sys.argv[1]
    path = os.path.join(root, "elsa", "generators", "tests", "test_Phantoms.cpp")
    src = open(path).read()
    at = src.index('TEST_CASE_TEMPLATE("Phantoms: Drawing a 2d Shepp-Logan phantom"')
    start = src.index("expected({{", at) + len("expected({{")
    end = src.index("}});", start)
    body = re.sub(r"//[^\n]*", "", src[start:end])
    vals = [float(v) for v in re.findall(r"[-+]?\d*\.?\d+(?:[eE][-+]?\d+)?", body)]
    assert len(vals) == 256, len(vals)
    out = os.path.join(HERE, "shepp_logan_2d_16.json")
    with open(out, "w") as f:
        json.dump({"source": "elsa generators/tests/test_Phantoms.cpp:145-187 (x fastest)",
                   "size": [16, 16], "values": vals}, f)
    print(out)


if __name__ == "__main__":
    main()
