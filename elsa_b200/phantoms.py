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
        img = np.zeros((n, n), np.float32)
        for amp, (cx, cy), (a, b), ang in MODIFIED_SHEPP_LOGAN_2D:
            center = (_scale_shift(n, cx), _scale_shift(n, cy))
            draw_filled_ellipse_2d(img, amp, center, (_scale(n, a), _scale(n, b)), ang)
        return img
    raise ValueError("phantom::modifiedSheppLogan: only 2d or 3d supported")


def _trunc_div(a, b):
    """C++ integer division (truncation toward zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _sheared_line_pairs(img, amp, center, x_off, y_off, shear):
    """One pair of horizontal lines of a sheared ellipse (EllipseGenerator.cpp:118-158), with the
    y axis flipped as the reference draws it."""
    ny, nx = img.shape
    for x in range(center[0] - x_off, center[0] + x_off + 1):
        shear_term = _trunc_div((x - center[0]) * shear[1], shear[0])
        for sgn in ((1, -1) if y_off != 0 else (1,)):
            y = ny - (center[1] + sgn * y_off + shear_term)
            if not (0 <= x < nx and 0 <= y < ny):
                raise ValueError("EllipseGenerator: drawing coordinate out of bounds")
            img[y, x] = np.float32(img[y, x] + np.float32(amp))


def _sheared_filled_ellipse(img, amp, center, sizes, shear):
    """Midpoint ellipse rasterisation in integer arithmetic, filled with horizontal line pairs
    (EllipseGenerator.cpp:50-116)."""
    sx, sy = sizes
    two_xx, two_yy = 2 * sx * sx, 2 * sy * sy
    # first part: y advances every step
    x, y = sx, 0
    x_change, y_change = sy * sy * (1 - 2 * sx), sx * sx
    err, x_stop, y_stop = 0, two_yy * sx, 0
    while x_stop >= y_stop:
        _sheared_line_pairs(img, amp, center, x, y, shear)
        y += 1
        y_stop += two_xx
        err += y_change
        y_change += two_xx
        if 2 * err + x_change > 0:
            x -= 1
            x_stop -= two_yy
            err += x_change
            x_change += two_yy
    # second part: x advances every step; a line pair is drawn whenever y changes
    x, y = 0, sy
    x_change, y_change = sy * sy, sx * sx * (1 - 2 * sy)
    err, x_stop, y_stop = 0, 0, two_xx * sy
    while x_stop < y_stop:
        x += 1
        x_stop += two_yy
        err += x_change
        x_change += two_yy
        if 2 * err + y_change > 0:
            _sheared_line_pairs(img, amp, center, x - 1, y, shear)
            y -= 1
            y_stop -= two_xx
            err += y_change
            y_change += two_xx


def draw_filled_ellipse_2d(img, amp, center, sizes, angle_deg):
    """Adds `amp` to the pixels of a filled ellipse (EllipseGenerator::drawFilledEllipse2d,
    generators/EllipseGenerator.cpp:10-48): integer centre and half axes; a rotation is turned
    into a shear of the axis-aligned rasterisation. img: float32 (ny, nx), x fastest."""
    sx, sy = int(sizes[0]), int(sizes[1])
    if sx == 0 and sy == 0:
        return
    ang = float(np.float32(angle_deg))
    if sx == sy or math.fmod(ang, 180.0) == 0:
        _sheared_filled_ellipse(img, amp, center, (sx, sy), (1, 0))
        return
    rad = ang * math.pi / 180.0
    theta = math.atan2(float(np.float32(-sy)) * math.tan(rad), float(sx))
    s0 = int(math.floor(float(np.float32(sx)) * math.cos(theta) * math.cos(rad)
                        - float(np.float32(sy)) * math.sin(theta) * math.sin(rad)))
    s1 = int(math.floor(float(np.float32(sx)) * math.cos(theta) * math.sin(rad)
                        + float(np.float32(sy)) * math.sin(theta) * math.cos(rad)))
    sheared = (abs(s0), _trunc_div(sy * sx, abs(s0)))
    _sheared_filled_ellipse(img, amp, center, sheared, (s0, s1))


def rectangle(shape, lower, upper):
    """phantoms::rectangle (generators/Phantoms.cpp:56-69): ones on [lower, upper) per axis.
    shape, lower, upper in elsa's axis order (x first); returns x-fastest C-order array."""
    img = np.zeros(tuple(reversed([int(s) for s in shape])), np.float32)
    sl = tuple(slice(int(lo), int(hi)) for lo, hi in zip(reversed(lower), reversed(upper)))
    img[sl] = 1.0
    return img


def circular(shape, radius):
    """phantoms::circular (generators/Phantoms.cpp:37-54): ones where |p - size/2| <= radius,
    p the integer voxel index (x first); returns x-fastest C-order array."""
    shape = [int(s) for s in shape]
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in reversed(shape)],
                        indexing="ij")
    d2 = np.zeros(grids[0].shape)
    for g, n in zip(grids, reversed(shape)):
        d2 += (g - np.float32(n) / np.float32(2.0)) ** 2
    return (np.sqrt(d2) <= radius).astype(np.float32)


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
