"""Known-answer cases re-expressed from elsa's own projector tests.

Each case gives the geometry (pose records built with the oracle's restatement of
core/Geometry.cpp), an input volume with the expected forward projection, and a sinogram with the
expected backprojection. Values are closed-form and come from the cited reference tests.
Volumes are numpy arrays indexed [z, y, x] / [y, x] (x fastest), as elsa's DataContainer(x, y, z).
"""
import math

import numpy as np

PI_F = float(np.float32(math.pi))
SQ3 = math.sqrt(3.0)


def _rad(deg):
    # Degree{d}.to_radian() = d * pi_t / 180 in float (core/StrongTypes.h:60)
    return float(np.float32(np.float32(deg) * np.float32(PI_F)) / np.float32(180))


def _pose2d(O, vol_dims, det_u, s2c, c2d, angle, cor=(0.0, 0.0), spacing=1.0):
    # VolumeData2D{Size2D, Spacing2D}: origin 0.5 * (size * spacing), core/StrongTypes.h:498-504
    sp = float(np.float32(spacing))
    vo = [0.5 * float(np.float32(v * sp)) for v in vol_dims]
    return O.geometry2d(s2c, c2d, angle, [sp, sp], vo, [1, 1], [0.5 * det_u, 0.5], 0.0, cor)


def _pose3d(O, vol_dims, det_uv, num_poses, s2c, c2d, gamma, beta=0.0, cor=(0.0, 0.0, 0.0),
            spacing=1.0):
    sp = float(np.float32(spacing))
    vo = [0.5 * float(np.float32(v * sp)) for v in vol_dims]
    so = [0.5 * det_uv[0], 0.5 * det_uv[1]]
    return O.geometry3d(s2c, c2d, [sp, sp, sp], vo, [1, 1], so, gamma, beta, 0.0, [0.0, 0.0],
                        cor)


def joseph_cases(O):
    """projectors/tests/test_JosephsMethod.cpp"""
    cases = []
    # :17-204 single ray through a 5x5 volume of ones at 0/180/90/270 degrees
    for deg, axis in ((0, "col"), (180, "col"), (90, "row"), (270, "row")):
        poses = _pose2d(O, (5, 5), 1, 100.0, 5.0, _rad(deg))[None]
        x = np.ones((5, 5), np.float32)
        bp = np.zeros((5, 5), np.float32)
        if axis == "col":
            bp[:, 2] = 5
        else:
            bp[2, :] = 5
        cases.append(dict(name="joseph_single_ray_%d" % deg, vol=(5, 5), det=(1, 1),
                          poses=poses, x=x, y_expect=np.array([5.0]), y=np.array([5.0]),
                          bp_expect=bp))
    # :1151-1214 x-, y- and z-axis aligned rays through a 3^3 volume
    beta = [0.0, 0.0, 0.0, 0.0, PI_F / 2, 3 * PI_F / 2]
    gamma = [0.0, PI_F, PI_F / 2, 3 * PI_F / 2, PI_F / 2, 3 * PI_F / 2]
    poses = np.stack([_pose3d(O, (3, 3, 3), (1, 1), 6, 60.0, 3.0, float(np.float32(g)),
                              float(np.float32(b))) for g, b in zip(gamma, beta)])
    x = np.zeros((3, 3, 3), np.float32)
    for i in range(3):
        x[1, 1, i] = 1
        x[1, i, 1] = 1
        x[i, 1, 1] = 1
    bp = np.array([0, 0, 0, 0, 6, 0, 0, 0, 0, 0, 6, 0, 6, 18, 6, 0, 6, 0, 0, 0, 0, 0, 6, 0, 0, 0,
                   0], np.float32).reshape(3, 3, 3)
    cases.append(dict(name="joseph_axis_aligned_3d", vol=(3, 3, 3), det=(1, 1, 6), poses=poses,
                      x=x, y_expect=np.full(6, 3.0), y=np.full(6, 3.0), bp_expect=bp))
    # :1217-1270 non-cubic volume 5x1x2, ray through the shorter dimension
    poses = _pose3d(O, (5, 1, 2), (1, 1), 1, 100.0, 5.0, 0.0, 0.0, (1.6, 0.0, 0.0))[None]
    x = np.zeros((2, 1, 5), np.float32)
    x[0, 0, 4] = 1
    x[1, 0, 4] = 1
    bp = np.zeros((2, 1, 5), np.float32)
    bp[0, 0, 4] = bp[1, 0, 4] = 0.6
    bp[0, 0, 3] = bp[1, 0, 3] = 0.4
    cases.append(dict(name="joseph_non_cubic", vol=(5, 1, 2), det=(1, 1, 1), poses=poses, x=x,
                      y_expect=np.array([1.2]), y=np.array([1.0]), bp_expect=bp))
    # :1273-1348 30 degree ray through the centre of a 4x4 volume
    poses = _pose2d(O, (4, 4), 1, 80.0, 4.0, -PI_F / 6)[None]
    w = 2 / math.sqrt(3.0)
    x = np.zeros((4, 4), np.float32)
    for (i, j) in ((3, 0), (1, 1), (1, 2), (1, 3)):
        x[j, i] = 1
    exp = np.array([0, 0, (3 - SQ3) / 2, (SQ3 - 1) / 2, 0, (SQ3 - 1) / (2 * SQ3),
                    (SQ3 + 1) / (2 * SQ3), 0, 0, (SQ3 + 1) / (2 * SQ3), (SQ3 - 1) / (2 * SQ3), 0,
                    (SQ3 - 1) / 2, (3 - SQ3) / 2, 0, 0]) * w
    cases.append(dict(name="joseph_30deg_center", vol=(4, 4), det=(1, 1), poses=poses, x=x,
                      y_expect=np.array([2 * w]), y=np.array([1.0]),
                      bp_expect=exp.reshape(4, 4)))
    # :1350-1390 30 degree ray through a single pixel
    poses = _pose2d(O, (4, 4), 1, 80.0, 4.0, -PI_F / 6, (-2 - SQ3 / 2, 0.0))[None]
    x = np.zeros((4, 4), np.float32)
    x[0, 0] = 1
    bp = np.zeros((4, 4), np.float32)
    bp[0, 0] = 1 / SQ3
    cases.append(dict(name="joseph_30deg_single_pixel", vol=(4, 4), det=(1, 1), poses=poses, x=x,
                      y_expect=np.array([1 / SQ3]), y=np.array([1.0]), bp_expect=bp,
                      tol=1e-4))
    return cases


def siddon_cases(O):
    """projectors/tests/test_SiddonsMethod.cpp"""
    cases = []
    # :1166-1227 30 degree ray through the centre of a 4x4 volume
    poses = _pose2d(O, (4, 4), 1, 80.0, 4.0, -PI_F / 6)[None]
    x = np.zeros((4, 4), np.float32)
    x[0, 3], x[0, 2], x[1, 2] = 1, 2, 3
    exp = np.array([0, 0, 2 - 2 / SQ3, 4 / SQ3 - 2, 0, 0, 2 / SQ3, 0, 0, 2 / SQ3, 0, 0,
                    4 / SQ3 - 2, 2 - 2 / SQ3, 0, 0])
    cases.append(dict(name="siddon_30deg_center", vol=(4, 4), det=(1, 1), poses=poses, x=x,
                      y_expect=np.array([2 * SQ3 + 2]), y=np.array([1.0]),
                      bp_expect=exp.reshape(4, 4)))
    # :1094-1141 x-, y- and z-axis aligned rays through a 3^3 volume
    beta = [0.0, 0.0, 0.0, 0.0, PI_F / 2, 3 * PI_F / 2]
    gamma = [0.0, PI_F, PI_F / 2, 3 * PI_F / 2, PI_F / 2, 3 * PI_F / 2]
    poses = np.stack([_pose3d(O, (3, 3, 3), (1, 1), 6, 60.0, 3.0, float(np.float32(g)),
                              float(np.float32(b))) for g, b in zip(gamma, beta)])
    x = np.zeros((3, 3, 3), np.float32)
    for i in range(3):
        x[1, 1, i] = 1
        x[1, i, 1] = 1
        x[i, 1, 1] = 1
    bp = np.array([0, 0, 0, 0, 6, 0, 0, 0, 0, 0, 6, 0, 6, 18, 6, 0, 6, 0, 0, 0, 0, 0, 6, 0, 0, 0,
                   0], np.float32).reshape(3, 3, 3)
    cases.append(dict(name="siddon_axis_aligned_3d", vol=(3, 3, 3), det=(1, 1, 6), poses=poses,
                      x=x, y_expect=np.full(6, 3.0), y=np.full(6, 3.0), bp_expect=bp))
    return cases


def binary_cases(O):
    """projectors/tests/test_BinaryMethod.cpp: one ray through a 5x5 volume of ones (source to
    centre 100, centre to detector 5) at several angles; y = A x and bp = A^T y = A^T A x."""
    cases = []
    ones = np.ones((5, 5), np.float32)
    column = np.zeros((5, 5), np.float32)
    column[:, 2] = 5
    row = np.zeros((5, 5), np.float32)
    row[2, :] = 5
    # :25-240 (cmp vectors in DataContainer order, x fastest)
    diag45 = np.array([9, 0, 0, 0, 0, 9, 9, 0, 0, 0, 0, 9, 9, 0, 0, 0, 0, 9, 9, 0, 0, 0, 0, 9, 9],
                      np.float32).reshape(5, 5)
    diag225 = np.array([9, 9, 0, 0, 0, 0, 9, 9, 0, 0, 0, 0, 9, 9, 0, 0, 0, 0, 9, 9, 0, 0, 0, 0,
                        9], np.float32).reshape(5, 5)
    for name, angle, y, bp in (("0deg", 0.0, 5.0, column), ("180deg", _rad(180), 5.0, column),
                               ("90deg", _rad(90), 5.0, row), ("270deg", _rad(270), 5.0, row),
                               ("45deg", _rad(45), 9.0, diag45),
                               ("225deg", _rad(225), 9.0, diag225)):
        poses = _pose2d(O, (5, 5), 1, 100.0, 5.0, angle)[None]
        cases.append(dict(name="binary_" + name, vol=(5, 5), det=(1, 1), poses=poses, x=ones,
                          y_expect=np.array([y]), y=np.array([y]), bp_expect=bp))
    # :242-325 one ray, four angles
    poses = np.stack([_pose2d(O, (5, 5), 1, 100.0, 5.0, a)
                      for a in (_rad(0), _rad(90), _rad(180), _rad(270))])
    cross = np.array([0, 0, 10, 0, 0, 0, 0, 10, 0, 0, 10, 10, 20, 10, 10, 0, 0, 10, 0, 0, 0, 0,
                      10, 0, 0], np.float32).reshape(5, 5)
    cases.append(dict(name="binary_4angles", vol=(5, 5), det=(1, 4), poses=poses, x=ones,
                      y_expect=np.full(4, 5.0), y=np.full(4, 5.0), bp_expect=cross))
    return cases


def lut_cases(O):
    """projectors/tests/test_LutProjector.cpp: the ray-driven blob projector (radius 2, alpha
    10.83, order 2) on 5x5 / 5^3 volumes, source to centre 100, centre to detector 5. Each case
    gives the expected detector values as multiples of the blob's weight at given distances and
    the relative tolerance of the reference check."""
    lut = O.blob_lut()

    def w(d):
        return float(O.lut_lerp(lut, 2.0, float(np.float32(d))))

    cases = []
    # :156-200 centre voxel, one ray, angles 0, 4, ..., 356 degrees
    x = np.zeros((5, 5), np.float32)
    x[2, 2] = 1
    for a in range(0, 360, 4):
        poses = _pose2d(O, (5, 5), 1, 100.0, 5.0, _rad(a))[None]
        cases.append(dict(name="lut_center_%d" % a, vol=(5, 5), det=(1, 1), poses=poses, x=x,
                          y_expect=np.array([w(0)]), tol=1.2e-5))
    # :203-249 two rays, :252-306 three rays
    for a in range(0, 360, 4):
        poses = _pose2d(O, (5, 5), 2, 100.0, 5.0, _rad(a))[None]
        cases.append(dict(name="lut_two_%d" % a, vol=(5, 5), det=(2, 1), poses=poses, x=x,
                          y_expect=np.array([w(0.4761878)] * 2), tol=0.01))
    for a in range(0, 360, 5):
        poses = _pose2d(O, (5, 5), 3, 100.0, 5.0, _rad(a))[None]
        cases.append(dict(name="lut_three_%d" % a, vol=(5, 5), det=(3, 1), poses=poses, x=x,
                          y_expect=np.array([w(0.95233786), w(0), w(0.95233786)]), tol=0.01))
    # :309-720 stepping of single rays (arrays indexed [y, x] = x(x, y) of the reference)
    step = [(0, [(2, j) for j in range(5)], 5 * w(0), 1.2e-5),
            (0, [(3, j) for j in range(5)], 5 * w(1), 1.2e-5),
            (0, [(1, j) for j in range(5)], 5 * w(1), 1.2e-5),
            (0, [(4, j) for j in range(5)], 5 * w(2), 1.2e-5),
            (0, [(0, j) for j in range(5)], 5 * w(2), 1.2e-5),
            (45, [(i, i) for i in range(5)], 5 * w(0), 1.2e-5),
            (45, [(0, 1), (1, 2), (2, 3), (3, 4)], 4 * w(0.707106769084930), 0.01),
            (45, [(1, 0), (2, 1), (3, 2), (4, 3)], 4 * w(0.707106769084930), 0.01),
            (45, [(0, 2), (1, 3), (2, 4)], 3 * w(2 * 0.707106769084930), 1.2e-5),
            (45, [(2, 0), (3, 1), (4, 2)], 3 * w(2 * 0.707106769084930), 1.2e-5),
            (90, [(i, 2) for i in range(5)], 5 * w(0), 1.2e-5),
            (90, [(i, 3) for i in range(5)], 5 * w(1), 1.2e-5)]
    for k, (a, vox, val, tol) in enumerate(step):
        xs = np.zeros((5, 5), np.float32)
        for (i, j) in vox:
            xs[j, i] = 1
        poses = _pose2d(O, (5, 5), 1, 100.0, 5.0, _rad(a))[None]
        cases.append(dict(name="lut_step_%d_%d" % (a, k), vol=(5, 5), det=(1, 1), poses=poses,
                          x=xs, y_expect=np.array([val]), tol=tol))
    # :110-153 3D: centre voxel of a 5^3 volume, Gamma of 0, 4, ..., 356 (radian)
    x3 = np.zeros((5, 5, 5), np.float32)
    x3[2, 2, 2] = 1
    for a in range(0, 360, 4):
        poses = _pose3d(O, (5, 5, 5), (1, 1), 1, 100.0, 5.0, float(np.float32(a)))[None]
        cases.append(dict(name="lut_center3d_%d" % a, vol=(5, 5, 5), det=(1, 1, 1), poses=poses,
                          x=x3, y_expect=np.array([w(0)]), tol=1.2e-5))
    return cases


def voxel_cases(O):
    """projectors/tests/test_BlobVoxelProjector.cpp:25-244: a centre voxel set to 1, projected
    onto one, two or three detector pixels. Expected values are blob LUT weights at the stated
    distances (op.blob(d) is the projected-blob LUT at d); tolerances are the reference's."""
    lut, support, _ = O.voxel_lut("blob", 3)
    lut2, support2, _ = O.voxel_lut("blob", 2)
    w = lambda d: O.lut_lerp(lut, support, d)  # noqa: E731
    cases = []
    # :25-71 3D, 5^3 volume, one pixel, spacings 0.5/1/1.5, gamma = 0..356 (radians, as written)
    for i in (1, 2, 3):
        sp = i / 2.0
        for ang in range(0, 360, 4):
            poses = _pose3d(O, (5, 5, 5), (1, 1), 1, 100.0, 5.0, float(np.float32(ang)),
                            spacing=sp)[None]
            x = np.zeros((5, 5, 5), np.float32)
            x[2, 2, 2] = 1
            cases.append(dict(name="blob3d_1px_sp%g_g%d" % (sp, ang), dim=3, vol=(5, 5, 5),
                              det=(1, 1, 1), poses=poses, x=x, y_expect=np.array([w(0.0)]),
                              rtol=0.005))
    # :74-121 2D, 5^2 volume, one pixel, spacings 0.5/1/1.5, Degree{0..356}
    for i in (1, 2, 3):
        sp = i / 2.0
        for ang in range(0, 360, 4):
            poses = _pose2d(O, (5, 5), 1, 100.0, 5.0, _rad(ang), spacing=sp)[None]
            x = np.zeros((5, 5), np.float32)
            x[2, 2] = 1
            cases.append(dict(name="blob2d_1px_sp%g_a%d" % (sp, ang), dim=2, vol=(5, 5),
                              det=(1, 1), poses=poses, x=x,
                              y_expect=np.array([O.lut_lerp(lut2, support2, 0.0)]), rtol=1e-5))
    # :124-170 2D, two pixels: both at distance 0.4761878 (1 % tolerance)
    for ang in range(0, 360, 4):
        poses = _pose2d(O, (5, 5), 2, 100.0, 5.0, _rad(ang))[None]
        x = np.zeros((5, 5), np.float32)
        x[2, 2] = 1
        v = O.lut_lerp(lut2, support2, 0.4761878)
        cases.append(dict(name="blob2d_2px_a%d" % ang, dim=2, vol=(5, 5), det=(2, 1),
                          poses=poses, x=x, y_expect=np.array([v, v]), rtol=0.01))
    # :173-244 2D, three pixels in 5 degree steps: centre weight(0), outer weight(0.95233786)
    for ang in range(0, 360, 5):
        poses = _pose2d(O, (5, 5), 3, 100.0, 5.0, _rad(ang))[None]
        x = np.zeros((5, 5), np.float32)
        x[2, 2] = 1
        v0 = O.lut_lerp(lut2, support2, 0.0)
        v1 = O.lut_lerp(lut2, support2, 0.95233786)
        cases.append(dict(name="blob2d_3px_a%d" % ang, dim=2, vol=(5, 5), det=(3, 1),
                          poses=poses, x=x, y_expect=np.array([v1, v0, v1]),
                          rtol=np.array([0.01, 1e-5, 0.01])))
    return cases
