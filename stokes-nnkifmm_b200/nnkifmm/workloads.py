"""Seeded synthetic workloads with the shapes of the benchmark configurations.

matvec_at_scale: 250k force points (half uniform in [0,1]^3, half on the
surfaces of 20 spheres with centres U[0.2,0.8]^3 and radii U[0.05,0.2]) and
1M quadrature points drawn the same way on the same spheres; forces
N(0,1); eps = 1e-3, mu = 1, nodeCapacity 64, p = 6.
sphere: the single-sphere mobility case (Sphere(1,[0 0 0],10) force nodes,
Sphere(...,40) quadrature, eps = 0.01, nodeCapacity 60).
two_squirmers_wall: two squirmers of radius 1 with centres 2.5 apart above a
triangular-lattice wall (Data Generation/Squiremers.m with a wall added).
"""
import numpy as np


def cube_sphere(r, centre, n):
    """Cube-surface lattice projected radially onto a sphere, n points per edge
    (the construction of Geometries/Sphere.m, n^3-(n-2)^3 points)."""
    lin = np.linspace(-r, r, n)
    k, i, j = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    j, i, k = j.ravel(), i.ravel(), k.ravel()
    shell = (j == 0) | (j == n - 1) | (i == 0) | (i == n - 1) | (k == 0) | (k == n - 1)
    X, Y, Z = lin[i[shell]], lin[j[shell]], lin[k[shell]]
    az = np.arctan2(Y, X)
    el = np.arctan2(Z, np.sqrt(X ** 2 + Y ** 2))
    return np.stack([r * np.cos(el) * np.cos(az) + centre[0], r * np.cos(el) * np.sin(az) + centre[1],
                     r * np.sin(el) + centre[2]], axis=1)


def squirmer_slip(points, B1, B2=0.0):
    """Tangential squirmer slip (B1 sin t + B2 sin t cos t) e_t on body-frame
    surface points, t the polar angle from the swimming axis z.  B1 alone is
    the reference's form (Data Generation/FlowField.m:39-49); B2 adds the
    pusher/puller mode."""
    p = np.asarray(points, float)
    x, y, z = p[:, 0], p[:, 1], p[:, 2]
    rho = np.hypot(x, y)
    r = np.sqrt(x * x + y * y + z * z)
    out = np.zeros_like(p)
    m = rho > 0
    # e_t = (x z, y z, -rho^2) / (r rho)
    et = np.stack([x[m] * z[m], y[m] * z[m], -rho[m] ** 2], axis=1) / (r[m] * rho[m])[:, None]
    st, ct = rho[m] / r[m], z[m] / r[m]
    out[m] = ((B1 * st + B2 * st * ct))[:, None] * et
    return out


def wall_lattice(n, spacing, z):
    """n x n triangular lattice in the plane z, centred at the origin (rows
    spacing*sqrt(3)/2 apart, every other row shifted by spacing/2)."""
    ix, iy = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    x = (ix + 0.5 * (iy % 2)) * spacing
    y = iy * spacing * np.sqrt(3) / 2
    pts = np.stack([x.ravel(), y.ravel(), np.full(ix.size, float(z))], axis=1)
    pts[:, :2] -= pts[:, :2].mean(axis=0)
    return pts


def two_squirmers_wall(edge_force=12, edge_quad=48, wall_n=200, spacing=0.05, B1=1.0, B2=0.5):
    """Two force- and torque-free squirmers (radius 1, centres (+-1.25, 0, 0),
    swimming axis z) with slip (B1, B2), above a wall z = -1.5 of wall_n^2
    lattice points whose force and quadrature points coincide (NN = I, as
    Data Generation/Squiremers.m:19-20), wall velocity 0."""
    body = cube_sphere(1.0, (0, 0, 0), edge_force)
    fine = cube_sphere(1.0, (0, 0, 0), edge_quad)
    wall = wall_lattice(wall_n, spacing, -1.5)
    return dict(body=body, fine=fine, slip=squirmer_slip(body, B1, B2), centres=[(-1.25, 0, 0), (1.25, 0, 0)],
                wall=wall)


def mixed_cloud(rng, n, centres, radii):
    u = rng.random((n // 2, 3))
    d = rng.standard_normal((n - n // 2, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    k = rng.integers(0, len(centres), n - n // 2)
    return np.concatenate([u, centres[k] + radii[k, None] * d])


def matvec_at_scale(n_force=250_000, n_quad=1_000_000, n_spheres=20, seed=20261204):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, (n_spheres, 3))
    radii = rng.uniform(0.05, 0.2, n_spheres)
    coarse = mixed_cloud(rng, n_force, centres, radii)
    fine = mixed_cloud(rng, n_quad, centres, radii)
    forces = rng.standard_normal((n_force, 3))
    return dict(coarse=coarse, fine=fine, forces=forces, eps=1e-3, mu=1.0, cap=64)


def prolate_spheroid(a, c, h):
    """Rings of spacing ~h on a prolate spheroid (minor a, major c), poles
    first: the construction of Geometries/prolateSpheroid.m."""
    pts = [np.array([[0.0, 0.0, c], [0.0, 0.0, -c]])]
    vN = int(np.ceil(np.pi * (3 * (a + c) - np.sqrt((3 * a + c) * (a + 3 * c))) / (2 * h)))
    for v in np.linspace(0.0, np.pi, vN)[1:-1]:
        z = c * np.cos(v)
        uN = int(np.ceil(2 * np.pi * a * np.sqrt(max(0.0, 1 - (z / c) ** 2)) / h))
        u = np.linspace(0.0, 2 * np.pi, uN + 1)[1:]
        pts.append(np.stack([a * np.cos(u) * np.sin(v), a * np.sin(u) * np.sin(v), np.full(uN, z)], axis=1))
    return np.concatenate(pts, axis=0)


def _spacing_for_count(a, c, target):
    lo, hi = 1e-4, 2.0
    for _ in range(60):  # the point count decreases with h
        mid = np.sqrt(lo * hi)
        if len(prolate_spheroid(a, c, mid)) > target:
            lo = mid
        else:
            hi = mid
    return hi


def batched_bodies(n_bodies=64, seed=20261206, nmin=2000, nmax=40000):
    """Independent rigid prolate spheroids: aspect U[1,5] at equal volume
    (a = aspect^-1/3, c = aspect^2/3), force-node count U[nmin, nmax] by
    bisection on the ring spacing h, quadrature at h/4 (about 16x), uniform
    random orientation.  Returns a list of (force points, quadrature points)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_bodies):
        asp = rng.uniform(1.0, 5.0)
        a, c = asp ** (-1.0 / 3.0), asp ** (2.0 / 3.0)
        h = _spacing_for_count(a, c, int(rng.uniform(nmin, nmax)))
        q, r = np.linalg.qr(rng.standard_normal((3, 3)))
        R = q * np.sign(np.diag(r))
        if np.linalg.det(R) < 0:
            R[:, 0] = -R[:, 0]
        coarse = prolate_spheroid(a, c, h) @ R.T
        fine = prolate_spheroid(a, c, h / 4) @ R.T
        out.append((coarse, fine))
    return out


def sphere_problem():
    """The single rigid sphere: Sphere(1,[0 0 0],10) force nodes and Sphere(1,[0 0 0],40)
    quadrature nodes; eps = 0.01, mu = 1, nodeCapacity 60."""
    return dict(coarse=cube_sphere(1.0, (0, 0, 0), 10), fine=cube_sphere(1.0, (0, 0, 0), 40), eps=0.01, mu=1.0,
                cap=60)
