"""The seeded benchmark workloads have the stated shapes: the single sphere
(488 / 9128 points, the oracle's Sphere construction), the two squirmers above
a wall (2 x 728 / 2 x 13,256 points, a 40,000-point wall), the matvec cloud
(half uniform in the unit cube, half on 20 sphere surfaces) and the batched
prolate spheroids (equal volume, aspect 1-5, 2k-40k force points, ~16x
quadrature, proper rotations)."""
import numpy as np

from nnkifmm import workloads as wl
from oracle.geometry import sphere


def test_single_sphere_matches_the_oracle_construction():
    s = wl.sphere_problem()
    assert s["coarse"].shape == (488, 3) and s["fine"].shape == (9128, 3)
    assert np.allclose(s["coarse"], sphere(1.0, [0, 0, 0], 10), rtol=0, atol=1e-14)
    assert np.allclose(s["fine"], sphere(1.0, [0, 0, 0], 40), rtol=0, atol=1e-14)
    assert np.allclose(np.linalg.norm(s["fine"], axis=1), 1.0)


def test_two_squirmers_above_a_wall():
    c = wl.two_squirmers_wall()
    assert c["body"].shape == (728, 3) and c["fine"].shape == (13256, 3) and c["wall"].shape == (40000, 3)
    assert np.all(c["wall"][:, 2] == -1.5) and np.allclose(c["wall"][:, :2].mean(axis=0), 0.0)
    # slip is tangential, zero at the poles, B1 at the equator
    s = c["slip"]
    assert np.abs(np.sum(s * c["body"], axis=1)).max() < 1e-12
    eq = np.abs(c["body"][:, 2]) < 1e-12
    assert np.allclose(np.linalg.norm(s[eq], axis=1), 1.0)


def test_matvec_cloud_halves():
    w = wl.matvec_at_scale(20_000, 80_000)
    for pts, n in ((w["coarse"], 20_000), (w["fine"], 80_000)):
        assert pts.shape == (n, 3)
        cube = pts[: n // 2]
        assert cube.min() >= 0.0 and cube.max() <= 1.0
    rng = np.random.default_rng(20261204)  # the generator's own draws: centres, then radii
    centres = rng.uniform(0.2, 0.8, (20, 3))
    radii = rng.uniform(0.05, 0.2, 20)
    surf = w["coarse"][10_000:]
    d = np.abs(np.linalg.norm(surf[:, None, :] - centres[None], axis=2) - radii[None])
    assert d.min(axis=1).max() < 1e-12  # every surface point lies on one of the spheres
    assert w["forces"].shape == (20_000, 3) and (w["eps"], w["cap"]) == (1e-3, 64)


def test_batched_prolate_spheroids():
    bodies = wl.batched_bodies(n_bodies=4)
    for coarse, fine in bodies:
        assert 1800 <= len(coarse) <= 40_000
        assert 10 <= len(fine) / len(coarse) <= 20
        # principal axes of the point cloud: one long axis c, two short a, a^2 c = 1
        ev = np.sort(np.linalg.eigvalsh(np.cov(coarse.T)))
        assert ev[2] >= ev[1] * 0.99 and abs(ev[0] - ev[1]) < 0.05 * ev[1]
        ext = np.abs(coarse @ np.linalg.eigh(np.cov(coarse.T))[1]).max(axis=0)
        a, c = ext[0], ext[2]
        assert 0.9 <= c / a <= 5.1 and abs(a * a * c - 1.0) < 0.02
