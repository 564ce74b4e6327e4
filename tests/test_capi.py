"""C ABI checks that need no GPU: the library loads, exports every symbol of include/*.h, builds
geometry bit-identical to the oracle and rejects invalid arguments with elsa_status codes."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(elsa_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def capi():
    from elsa_b200 import build, _capi
    build.build()
    return _capi


def test_library_exports_header(capi):
    lib = capi.lib()
    declared = _declared_symbols()
    assert declared, "no declarations found"
    for name in sorted(declared):
        assert hasattr(lib, name), name
    # the ctypes table covers every declaration, and nothing undeclared
    assert declared == set(capi.SIGNATURES)


def _header_constants():
    """ELSA_* integer constants of include/*.h: #define values and enumerators."""
    consts = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for name, value in re.findall(r"#define\s+ELSA_([A-Z0-9_]+)\s+(-?\d+)\b", text):
            consts[name] = int(value)
        for name, value in re.findall(r"\bELSA_([A-Z0-9_]+)\s*=\s*(-?\d+)", text):
            consts[name] = int(value)
    return consts


def test_python_constants_match_header(capi):
    """Every constant the Python bindings mirror (projector and solver kinds, knobs, footprint
    modes, status codes, ...) has the header's value, and the knob names cover every knob."""
    consts = _header_constants()
    assert consts["KNOB_COUNT"] == capi.KNOB_COUNT == len(capi.KNOB_NAMES)
    mirrored = 0
    for name, value in consts.items():
        short = name[len("ERROR_"):] if name.startswith("ERROR_") else name
        for candidate in (name, short):
            if hasattr(capi, candidate) and isinstance(getattr(capi, candidate), int):
                assert getattr(capi, candidate) == value, name
                mirrored += 1
                break
    assert mirrored >= 25, mirrored
    for k, knob in enumerate(capi.KNOB_NAMES):
        assert consts["KNOB_" + knob.upper()] == k


def test_geometry_bit_identical_to_oracle(capi, oracle):
    for args in [([128, 128], 180, 360, 1000, 250, [182]),
                 ([256, 256, 256], 360, 360, 2560, 640, [384, 384]),
                 ([128, 128, 128], 180, 360, 1280, 320, [192, 192]),
                 ([64, 96, 80], 7, 200, 500, 100, None)]:
        po, do = oracle.circle_trajectory(*args)
        pp, dp = capi.circle_trajectory(*args)
        assert np.array_equal(do, dp)
        assert np.array_equal(po.view(np.uint32), pp.view(np.uint32))
    a = dict(vol_spacing=[1, 2, 0.5], vol_origin=[10, 9, 8], sino_spacing=[1.5, 0.7],
             sino_origin=[5, 6], gamma=0.3, beta=0.2, alpha=0.1, pp_offset=[0.5, -0.3],
             cor_offset=[0.1, 0.2, 0.3])
    po = oracle.geometry3d(100.0, 20.0, **a)
    pp = capi.pose_3d(100.0, 20.0, **a)
    assert np.array_equal(po.view(np.uint32), pp.view(np.uint32))
    po = oracle.geometry2d(100.0, 20.0, 0.7, [1, 1.5], [3, 4], [0.8, 1], [2, 1], 0.25, [0.5, -1])
    pp = capi.pose_2d(100.0, 20.0, 0.7, [1, 1.5], [3, 4], [0.8, 1], [2, 1], 0.25, [0.5, -1])
    assert np.array_equal(po.view(np.uint32), pp.view(np.uint32))


def test_invalid_arguments(capi):
    poses, det = capi.circle_trajectory([8, 8], 4, 360, 40, 10)
    with pytest.raises(capi.InvalidArgumentError):
        capi.Projector(capi.PROJECTOR_JOSEPH, [8, 8, 8, 8], det, poses)
    with pytest.raises(capi.InvalidArgumentError):
        capi.Projector(capi.PROJECTOR_JOSEPH, [8, 0], det, poses)
    with pytest.raises(capi.InvalidArgumentError):
        capi.circle_trajectory([8, 8, 8, 8], 4, 360, 40, 10)
    lib = capi.lib()
    h = ctypes.c_void_p()
    st = lib.elsa_projector_create(0, 2, None, None, None, None, 0, ctypes.byref(h))
    assert st == 1 and b"null" in lib.elsa_last_error()
    assert lib.elsa_projector_create(0, 2, None, None, None, None, 0, None) == 1
    assert lib.elsa_abi_version() == 1
