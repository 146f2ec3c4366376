"""Point generators of the reference (Geometries/*.m), used to build the
synthetic inputs of the parity tests and the benchmark.

Test infrastructure only (see oracle/__init__.py).  The product library takes
points as plain arrays; these generators only make inputs.
"""
import numpy as np

from .mlab import linspace, meshgrid3_colmajor


def sphere(r, centre, n):
    """Cube-surface lattice projected radially onto a sphere;
    Geometries/Sphere.m:15-43.  ``n`` points per cube edge give
    n^3 - (n-2)^3 points, in MATLAB meshgrid column-major order."""
    pos = linspace(-r, r, n)
    X, Y, Z, j, i, k = meshgrid3_colmajor(pos, pos, pos)
    interior = (j >= 1) & (j <= n - 2) & (i >= 1) & (i <= n - 2) & (k >= 1) & (k <= n - 2)
    X, Y, Z = X[~interior], Y[~interior], Z[~interior]
    az = np.arctan2(Y, X)
    el = np.arctan2(Z, np.sqrt(X ** 2 + Y ** 2))
    x = r * np.cos(el) * np.cos(az) + centre[0]
    y = r * np.cos(el) * np.sin(az) + centre[1]
    z = r * np.sin(el) + centre[2]
    return np.stack([x, y, z], axis=1)


def prolate_spheroid(a, c, h):
    """Rings of spacing ~h on a prolate spheroid (minor a, major c);
    Geometries/prolateSpheroid.m:14-28.  The two poles come first."""
    pts = [np.array([[0.0, 0.0, c], [0.0, 0.0, -c]])]
    vN = int(np.ceil(np.pi * (3 * (a + c) - np.sqrt((3 * a + c) * (a + 3 * c))) / (2 * h)))
    v = linspace(0.0, np.pi, vN)
    for i in range(1, vN - 1):
        z = c * np.cos(v[i])
        uN = int(np.ceil(2 * np.pi * a * np.sqrt(1 - (z / c) ** 2) / h))
        u = linspace(0.0, 2 * np.pi, uN + 1)[1:]
        x = a * np.cos(u) * np.sin(v[i])
        y = a * np.sin(u) * np.sin(v[i])
        pts.append(np.stack([x, y, np.full(uN, z)], axis=1))
    return np.concatenate(pts, axis=0)


def triangular_lattice(h, centre, limits):
    """Triangular lattice in a plane; Geometries/TriangularLattice.m:16-38."""
    v = np.sqrt(h ** 2 - (h / 2) ** 2)
    xl, yl = limits
    rows = []
    yc = 0.0
    disp = 0
    while yc < yl:
        if disp == 0:
            xx = np.arange(0.0, xl + 1e-12 * h, h)
            xx = xx[xx <= xl]
            disp = 1
        else:
            xx = np.arange(h / 2, xl + 1e-12 * h, h)
            xx = xx[xx <= xl]
            disp = 0
        rows.append(np.stack([xx, np.full(len(xx), yc)], axis=1))
        yc = yc + v
    g = np.concatenate(rows, axis=0)
    return g[:, 0] - xl / 2 + centre[0], g[:, 1] - yl / 2 + centre[1]


def wall_tri(centre, scale, axis, h):
    """Triangular-lattice plane normal to ``axis`` (1, 2, 3);
    Geometries/wallTri.m:14-22 (note the reference subtracts the centre on
    the in-plane axes)."""
    x1, x2 = triangular_lattice(h, (0.0, 0.0), scale)
    n = len(x1)
    if axis == 1:
        return np.stack([np.full(n, centre[0]), x1 - centre[1], x2 - centre[2]], axis=1)
    if axis == 2:
        return np.stack([x1 - centre[0], np.full(n, centre[1]), x2 - centre[2]], axis=1)
    return np.stack([x1 - centre[0], x2 - centre[1], np.full(n, centre[2])], axis=1)


def rotate(points, alpha, beta, gamma, centre):
    """Rx*Ry*Rz rotation about ``centre``; Geometries/Rotate.m:12-21."""
    p = np.asarray(points, dtype=np.float64) - np.asarray(centre)
    ca, sa, cb, sb, cg, sg = (np.cos(alpha), np.sin(alpha), np.cos(beta),
                              np.sin(beta), np.cos(gamma), np.sin(gamma))
    Rx = np.array([[1, 0, 0], [0, ca, sa], [0, -sa, ca]])
    Ry = np.array([[cb, 0, -sb], [0, 1, 0], [sb, 0, cb]])
    Rz = np.array([[cg, sg, 0], [-sg, cg, 0], [0, 0, 1]])
    R = Rx @ Ry @ Rz
    return (R @ p.T).T + np.asarray(centre)


def velocity_modes(points, vel, mom):
    """Rigid-body point velocities U + Omega x X; Geometries/velocityModes.m:13-25."""
    p = np.asarray(points, dtype=np.float64)
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    ux = vel[0] + mom[1] * z - mom[2] * y
    uy = vel[1] + mom[2] * x - mom[0] * z
    uz = vel[2] + mom[0] * y - mom[1] * x
    return np.stack([ux, uy, uz], axis=1)


def squirmer_slip(points, b1, b2=0.0):
    """Tangential squirmer slip (B1 sin(t) + B2 sin(t) cos(t)) e_theta.  The
    reference form has the B1 mode only (Data Generation/FlowField.m:39-49,
    ``scale*sin(theta).*tangent``); the B2 term is an extension."""
    p = np.asarray(points, dtype=np.float64)
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    rho = np.sqrt(x ** 2 + y ** 2)
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        tan = np.stack([x * z, y * z, -(x ** 2 + y ** 2)], axis=1) / (r * rho)[:, None]
        tan[np.isnan(tan)] = 0.0
        th = np.arccos(z / r)
    amp = b1 * np.sin(th) + b2 * np.sin(th) * np.cos(th)
    return amp[:, None] * tan


def random_rotation(rng):
    """Uniform random rotation matrix (QR of a Gaussian matrix, sign-fixed)."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q
