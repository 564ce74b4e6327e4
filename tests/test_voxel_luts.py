"""The product's voxel-projector lookup tables (host code behind elsa_voxel_lut, no GPU needed)
against the oracle restatement (bit for bit) and elsa's golden arrays."""
import json
import os

import numpy as np
import pytest

KINDS = {"blob": 2, "bspline": 3, "phase_blob": 4, "phase_bspline": 5}


@pytest.mark.parametrize("name", sorted(KINDS))
@pytest.mark.parametrize("dim", [2, 3])
def test_lut_matches_oracle_bitwise(oracle, name, dim):
    from elsa_b200 import _capi
    table, support = _capi.voxel_lut(KINDS[name], dim)
    ref, ref_support, _ = oracle.voxel_lut(name, dim)
    assert support == ref_support
    assert np.array_equal(table.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("order", [0, 1, 2, 3, 4])
def test_bspline_orders_match_oracle(oracle, order):
    from elsa_b200 import _capi
    for dim in (2, 3):
        table, _ = _capi.voxel_lut(KINDS["bspline"], dim, (float(order),))
        assert np.array_equal(table, oracle.bspline_lut(dim, order))


def test_lut_golden_arrays():
    """101-sample tables against test_Luts.cpp:125-305 (the reference checks lut(i/50) with
    epsilon 1e-6; the table entry i sits exactly at i/50)."""
    from elsa_b200 import _capi
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "voxel_luts.json")
    with open(path) as f:
        g = json.load(f)["luts"]
    blob, _ = _capi.voxel_lut(KINDS["blob"], 3, (2.0, 10.83, 2.0), 101)
    exp = np.array(g["projected_blob_lut_a2_alpha10.83_m2"])
    assert np.all(np.abs(blob[:99] - exp[:99]) < 1e-6 * (1 + np.abs(exp[:99])))
    spline, _ = _capi.voxel_lut(KINDS["bspline"], 2, (3.0,), 101)
    exp = np.array(g["projected_bspline_lut_order3_dim2"])
    assert np.all(np.abs(spline - exp) < 1e-6 * (1 + np.abs(exp)))


def test_lut_argument_errors():
    from elsa_b200 import _capi
    import elsa_b200
    with pytest.raises(elsa_b200.InvalidArgumentError):
        _capi.voxel_lut(KINDS["blob"], 3, (2.0, 10.83, 3.0))  # order 3 has no closed form
    with pytest.raises(elsa_b200.InvalidArgumentError):
        _capi.voxel_lut(KINDS["phase_blob"], 3, (2.0, 10.83, 0.0))
    with pytest.raises(elsa_b200.InvalidArgumentError):
        _capi.voxel_lut(KINDS["bspline"], 4)
