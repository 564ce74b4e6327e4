"""Input generators (elsa_b200.phantoms) against elsa's phantom tests
(generators/tests/test_Phantoms.cpp)."""
import json
import os

import numpy as np

from elsa_b200 import phantoms

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "shepp_logan_2d_16.json")


def test_shepp_logan_2d_golden():
    """test_Phantoms.cpp:145-187: the 16 x 16 modified Shepp-Logan, pixel by pixel."""
    with open(GOLDEN) as f:
        g = np.array(json.load(f)["values"])
    p = phantoms.modified_shepp_logan((16, 16)).ravel()
    np.testing.assert_allclose(p, g, rtol=0, atol=1e-6)


def test_rectangle():
    """test_Phantoms.cpp:22-91"""
    full = phantoms.rectangle((16, 16), (0, 0), (16, 16))
    assert np.all(full == 1)
    r = phantoms.rectangle((16, 16), (4, 4), (12, 12))
    assert r.sum() == 64 and np.all(r[4:12, 4:12] == 1)
    r3 = phantoms.rectangle((16, 16, 16), (4, 4, 4), (12, 12, 12))
    assert r3.sum() == 512 and np.all(r3[4:12, 4:12, 4:12] == 1)


def test_circular():
    """test_Phantoms.cpp:93-143: pixels with |p - size/2| <= r are 1, others 0."""
    for dim in (2, 3):
        shape = (16,) * dim
        for r in (1.0, 3.0, 5.5, 8.0):
            c = phantoms.circular(shape, r)
            for idx in np.ndindex(c.shape):
                d = np.sqrt(sum((i - 8.0) ** 2 for i in idx))
                assert c[idx] == (1.0 if d <= r else 0.0)


def test_shepp_logan_3d_properties():
    v = phantoms.modified_shepp_logan((64, 64, 64))
    assert v.shape == (64, 64, 64) and v.dtype == np.float32
    assert abs(v.max() - 1.0) < 1e-6 and v.min() > -1e-6
    assert v[32, 32, 32] > 0 and v[0, 0, 0] == 0


def test_seeded_generators():
    a = phantoms.random_ellipsoids(32, 20, seed=3)
    b = phantoms.random_ellipsoids(32, 20, seed=3)
    assert np.array_equal(a, b) and a.max() > 0
    n1 = phantoms.gaussian_noise((100,), 0.01, seed=1)
    assert np.array_equal(n1, phantoms.gaussian_noise((100,), 0.01, seed=1))
    assert abs(float(np.std(phantoms.gaussian_noise((100000,), 0.01, seed=2))) - 0.01) < 5e-4
