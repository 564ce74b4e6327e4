"""Input generators: modified Shepp-Logan phantoms, random ellipsoids, seeded noise.

These produce the synthetic inputs of the benchmarks and tests; they are not on the hot path.
Parameters follow elsa's generators/Phantoms.h:77-104 (3D table), Phantoms.cpp:89-120 (2D
ellipses) and the inside test of generators/Ellipsoid.cpp (integer voxel offsets from an integer
centre, ZXZ Euler rotation, generators/PhantomDefines.cpp:7-36). Arrays are returned in numpy C
order with x fastest: shape (ny, nx) in 2D and (nz, ny, nx) in 3D.
"""
import math

import numpy as np

# A, a, b, c, x0, y0, z0, phi, theta, psi
MODIFIED_SHEPP_LOGAN_3D = [
    (1.0, .6900, .920, .810, 0.00, 0.0, 0.0, 0.0, 0.0, 0.0),
    (-.8, .6624, .874, .780, 0.00, -.0184, 0.0, 0.0, 0.0, 0.0),
    (-.2, .1100, .310, .220, .22, 0.0, 0.0, -18.0, 0.0, 10.0),
    (-.2, .1600, .410, .280, -.22, 0.0, 0.0, 18.0, 0.0, 10.0),
    (.1, .2100, .250, .410, 0.00, .35, -.15, 0.0, 0.0, 0.0),
    (.1, .0460, .046, .050, 0.00, .1, .25, 0.0, 0.0, 0.0),
    (.1, .0460, .046, .050, 0.00, -.1, .25, 0.0, 0.0, 0.0),
    (.1, .0460, .023, .050, -.08, -.605, 0.0, 0.0, 0.0, 0.0),
    (.1, .0230, .023, .020, 0.00, -.606, 0.0, 0.0, 0.0, 0.0),
    (.1, .0230, .046, .020, .06, -.605, 0.0, 0.0, 0.0, 0.0),
]

# amplitude, (cx, cy), (a, b), angle in degrees
MODIFIED_SHEPP_LOGAN_2D = [
    (1.0, (0.0, 0.0), (.69, .92), 0.0),
    (-.8, (0.0, -.0184), (.6624, .8740), 0.0),
    (-.2, (.22, 0.0), (.11, .31), -18.0),
    (-.2, (-.22, 0.0), (.16, .41), 18.0),
    (.1, (0.0, .35), (.21, .25), 0.0),
    (.1, (0.0, .1), (.046, .046), 0.0),
    (.1, (0.0, -.1), (.046, .046), 0.0),
    (.1, (-.08, -.605), (.046, .023), 0.0),
    (.1, (0.0, -.606), (.023, .023), 0.0),
    (.1, (.06, -.605), (.023, .046), 0.0),
]


def _scale(n, v):
    return int(round(float(np.float32(v) * np.float32(n - 1) / np.float32(2.0))))


def _scale_shift(n, v):
    return int(round(float(v) * float(n - 1) / 2.0)) + n // 2


def _zxz(phi, theta, psi):
    p, t, s = (math.radians(a) for a in (phi, theta, psi))
    cp, sp, ct, st, cs, ss = (math.cos(p), math.sin(p), math.cos(t), math.sin(t), math.cos(s),
                              math.sin(s))
    return np.array([[cp * cs - ct * sp * ss, -cp * ss - ct * cs * sp, sp * st],
                     [cs * sp + cp * ct * ss, cp * ct * cs - sp * ss, -cp * st],
                     [st * ss, cs * st, ct]])


def _add_ellipsoid(vol, amp, center, half, eulers):
    nz, ny, nx = vol.shape
    a, b, c = (float(h) for h in half)
    if min(a, b, c) < 1 or amp == 0:
        return
    rot = _zxz(*eulers).T if any(e != 0 for e in eulers) else np.eye(3)
    r = int(math.ceil(max(a, b, c)))
    cx, cy, cz = center
    xs = np.arange(max(0, cx - r), min(nx, cx + r + 1))
    ys = np.arange(max(0, cy - r), min(ny, cy + r + 1))
    zs = np.arange(max(0, cz - r), min(nz, cz + r + 1))
    if not (len(xs) and len(ys) and len(zs)):
        return
    Z, Y, X = np.meshgrid(zs - cz, ys - cy, xs - cx, indexing="ij")
    d = np.stack([X, Y, Z]).reshape(3, -1).astype(np.float64)
    d = rot @ d
    inside = (d[0] ** 2 * (b * b * c * c) + d[1] ** 2 * (a * a * c * c) +
              d[2] ** 2 * (a * a * b * b)) <= a * a * b * b * c * c
    sub = vol[zs[0]:zs[-1] + 1, ys[0]:ys[-1] + 1, xs[0]:xs[-1] + 1]
    sub += (inside.reshape(sub.shape) * np.float32(amp)).astype(np.float32)


def modified_shepp_logan(shape):
    """Modified Shepp-Logan phantom, 2D (n, n) or 3D (n, n, n), float32, x fastest."""
    shape = tuple(int(s) for s in shape)
    if len(shape) == 3:
        n = shape[0]
        if not (shape[0] == shape[1] == shape[2]):
            raise ValueError("phantom::modifiedSheppLogan: 3d size has to be cubed")
        vol = np.zeros((n, n, n), np.float32)
        for e in MODIFIED_SHEPP_LOGAN_3D:
            half = (_scale(n, e[1]), _scale(n, e[2]), _scale(n, e[3]))
            center = (_scale_shift(n, e[4]), _scale_shift(n, e[5]), _scale_shift(n, e[6]))
            _add_ellipsoid(vol, e[0], center, half, e[7:10])
        return vol
    if len(shape) == 2:
        n = shape[0]
        if shape[0] != shape[1]:
            raise ValueError("phantom::modifiedSheppLogan: 2d size has to be square")
        img = np.zeros((n, n), np.float64)
        yy, xx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        for amp, (cx, cy), (a, b), ang in MODIFIED_SHEPP_LOGAN_2D:
            A, B = _scale(n, a), _scale(n, b)
            if A == 0 and B == 0:
                continue
            x0, y0 = _scale_shift(n, cx), _scale_shift(n, cy)
            t = math.radians(ang)
            dx = xx - x0
            # the reference draws with the y axis flipped (EllipseGenerator.cpp)
            dy = (n - yy) - y0
            u = dx * math.cos(t) + dy * math.sin(t)
            v = -dx * math.sin(t) + dy * math.cos(t)
            img += amp * ((u / max(A, 1e-9)) ** 2 + (v / max(B, 1e-9)) ** 2 <= 1.0)
        return img.astype(np.float32)
    raise ValueError("phantom::modifiedSheppLogan: only 2d or 3d supported")


def random_ellipsoids(n, count=20, seed=0):
    """n^3 volume of `count` seeded random ellipsoids with densities U(0,1), added together."""
    rng = np.random.default_rng(seed)
    vol = np.zeros((n, n, n), np.float32)
    for _ in range(count):
        amp = float(rng.uniform(0.0, 1.0))
        half = tuple(int(h) for h in rng.integers(max(2, n // 16), max(3, n // 4), 3))
        center = tuple(int(c) for c in rng.integers(n // 4, 3 * n // 4, 3))
        eulers = tuple(float(e) for e in rng.uniform(0.0, 180.0, 3))
        _add_ellipsoid(vol, amp, center, half, eulers)
    return vol


def gaussian_noise(shape, sigma, seed=0):
    """Seeded additive Gaussian noise (elsa's GaussianNoiseGenerator is unseeded,
    generators/NoiseGenerators.cpp:11-25)."""
    return (np.random.default_rng(seed).standard_normal(shape) * sigma).astype(np.float32)
