"""Generates the golden fixtures of tests/golden/*.npz from the FP64 oracle
(the CPU restatement of the reference under oracle/).

    python tests/golden/make_golden.py

Each fixture holds seeded inputs, the oracle's tree arrays and U/V/W/X lists
(1-based reference ids, flattened with offsets), and the oracle's KIFMM
outputs in the reference's own per-node-LU structure.  The GPU tests compare
the library against these files, so they run without the slow oracle.
"""
import os
import sys
import time

import numpy as np
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.geometry import sphere  # noqa: E402
from oracle.kernel import apply_kernel  # noqa: E402
from oracle.kifmm import KIFMM  # noqa: E402
from oracle.nearest import nearest_matrix  # noqa: E402
from oracle.octree import OcTree  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def lists_flat(tree):
    out = {}
    for name, L in zip("UVWX", [tree.U, tree.V, tree.W, tree.X]):
        off = np.zeros(tree.node_count + 1, np.int64)
        ids = []
        for i in range(1, tree.node_count + 1):
            ids.extend(int(v) for v in L[i])
            off[i] = len(ids)
        out[f"list_{name}_off"] = off
        out[f"list_{name}_ids"] = np.array(ids, np.int32)
    return out


def tree_arrays(tree):
    d = dict(level=tree.level[1:].astype(np.int32), parent=tree.parent[1:].astype(np.int32),
             children=tree.children[1:].astype(np.int32), corners=tree.corners[1:],
             point_index=tree.point_index.astype(np.int32))
    d.update(lists_flat(tree))
    return d


def nn_arrays(NN):
    NN = sp.csr_matrix(NN)
    NN.sort_indices()
    return dict(nn_indptr=NN.indptr.astype(np.int64), nn_indices=NN.indices.astype(np.int32),
                nn_data=NN.data.astype(np.float64))


def mixed_points(rng, n, nsph=3):
    u = rng.random((n // 2, 3))
    cen = rng.uniform(0.2, 0.8, (nsph, 3))
    rad = rng.uniform(0.05, 0.2, nsph)
    d = rng.standard_normal((n - n // 2, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    k = rng.integers(0, nsph, n - n // 2)
    return np.concatenate([u, cen[k] + rad[k, None] * d]), cen, rad


def sphere_case():
    """Rigid-sphere geometry: Sphere(1,[0 0 0],10) force nodes, Sphere(...,40) quadrature."""
    rng = np.random.default_rng(20261203)
    c = sphere(1.0, [0, 0, 0], 10)
    f = sphere(1.0, [0, 0, 0], 40)
    NN = nearest_matrix(c, f)
    tree = OcTree(c, c, node_capacity=60, nearest=1, fine_points=f, NN=NN)
    F = rng.standard_normal((len(c), 3))
    eps, mu = 0.01, 1.0
    fmm = KIFMM(tree, eps, mu)
    t = time.time()
    vel = fmm.compute_vel(F)
    vel4 = fmm.compute_vel_sparse(F)
    red = fmm.reduced_compute_vel(F)
    U = rng.standard_normal((len(c), 3))
    rsol = fmm.reduced_solve(U)
    direct = apply_kernel(f, c, NN @ F, eps, mu)
    print(f"sphere: {time.time() - t:.1f}s, fmm vs direct {np.linalg.norm(vel - direct) / np.linalg.norm(direct):.2e}")
    # eps-derivative of the reference operator: w^T (dF/deps) F by a central
    # difference of the oracle's per-node-LU passes (h = 1e-4 eps; 1e-3 gives
    # the same to 1e-8)
    wts = rng.standard_normal((len(c), 3))
    h = 1e-4 * eps
    vp = KIFMM(tree, eps + h, mu).compute_vel(F)
    vm = KIFMM(tree, eps - h, mu).compute_vel(F)
    deps_fd = float((wts * (vp - vm)).sum()) / (2 * h)
    d = dict(coarse=c, fine=f, F=F, U=U, eps=eps, mu=mu, cap=60, vel=vel, vel_sparse=vel4, reduced=red,
             reduced_solve=rsol, direct=direct, deps_w=wts, deps_fd=deps_fd)
    d.update(nn_arrays(NN))
    d.update(tree_arrays(tree))
    np.savez_compressed(os.path.join(OUT, "sphere10_40.npz"), **d)


def adaptive_plain_case():
    """Adaptive tree (uniform + sphere shells), plain mode, pot == tgt."""
    rng = np.random.default_rng(20261204)
    x, _, _ = mixed_points(rng, 1600)
    tree = OcTree(x, x, node_capacity=32)
    F = rng.standard_normal((len(x), 3))
    eps, mu = 1e-3, 1.0
    t = time.time()
    vel = KIFMM(tree, eps, mu).compute_vel(F)
    direct = apply_kernel(x, x, F, eps, mu)
    print(f"adaptive plain: {time.time() - t:.1f}s, nodes {tree.node_count}, "
          f"fmm vs direct {np.linalg.norm(vel - direct) / np.linalg.norm(direct):.2e}")
    d = dict(points=x, F=F, eps=eps, mu=mu, cap=32, vel=vel, direct=direct)
    d.update(tree_arrays(tree))
    np.savez_compressed(os.path.join(OUT, "adaptive_plain_1600.npz"), **d)


def adaptive_nearest_case():
    """Adaptive NEAREST tree: 1200 force points, 4x quadrature of the same mix."""
    rng = np.random.default_rng(20261205)
    c, cen, rad = mixed_points(rng, 1200)
    q = 4800
    u = rng.random((q // 2, 3))
    d = rng.standard_normal((q - q // 2, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    k = rng.integers(0, len(cen), q - q // 2)
    f = np.concatenate([u, cen[k] + rad[k, None] * d])
    NN = nearest_matrix(c, f)
    tree = OcTree(c, c, node_capacity=40, nearest=1, fine_points=f, NN=NN)
    F = rng.standard_normal((len(c), 3))
    eps, mu = 1e-3, 1.0
    t = time.time()
    vel = KIFMM(tree, eps, mu).compute_vel(F)
    direct = apply_kernel(f, c, NN @ F, eps, mu)
    print(f"adaptive nearest: {time.time() - t:.1f}s, nodes {tree.node_count}, "
          f"fmm vs direct {np.linalg.norm(vel - direct) / np.linalg.norm(direct):.2e}")
    dd = dict(coarse=c, fine=f, F=F, eps=eps, mu=mu, cap=40, vel=vel, direct=direct)
    dd.update(nn_arrays(NN))
    dd.update(tree_arrays(tree))
    np.savez_compressed(os.path.join(OUT, "adaptive_nearest_1200.npz"), **dd)


def split_case():
    """Sources != targets (OcTree(fine, targets)), plain mode."""
    rng = np.random.default_rng(20261206)
    src, _, _ = mixed_points(rng, 1500)
    tgt = rng.random((700, 3)) * 0.8 + 0.1
    tree = OcTree(src, tgt, node_capacity=24)
    F = rng.standard_normal((len(src), 3))
    eps, mu = 2e-3, 1.3
    t = time.time()
    vel = KIFMM(tree, eps, mu).compute_vel(F)
    direct = apply_kernel(src, tree.points[tree.targets], F, eps, mu)
    print(f"split: {time.time() - t:.1f}s, nodes {tree.node_count}, "
          f"fmm vs direct {np.linalg.norm(vel - direct) / np.linalg.norm(direct):.2e}")
    d = dict(src=src, tgt=tgt, F=F, eps=eps, mu=mu, cap=24, vel=vel, direct=direct,
             potentials=tree.potentials, targets=tree.targets, points=tree.points)
    d.update(tree_arrays(tree))
    np.savez_compressed(os.path.join(OUT, "split_1500_700.npz"), **d)


def matvec_case():
    """The matvec-at-scale distribution (50% uniform in the unit cube, 50% on
    20 spheres, NEAREST with 4x quadrature, eps = 1e-3, nodeCapacity 64) at
    4000 force / 16000 quadrature points, drawn by the same seeded generator
    as the 250k / 1M benchmark (nnkifmm/workloads.py, loaded on its own)."""
    import importlib.util
    path = os.path.join(ROOT, "stokes-nnkifmm_b200", "nnkifmm", "workloads.py")
    spec = importlib.util.spec_from_file_location("nnk_workloads_standalone", path)
    wl = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(wl)
    w = wl.matvec_at_scale(4000, 16000)
    c, f, F = w["coarse"], w["fine"], w["forces"]
    NN = nearest_matrix(c, f)
    tree = OcTree(c, c, node_capacity=w["cap"], nearest=1, fine_points=f, NN=NN)
    t = time.time()
    vel = KIFMM(tree, w["eps"], w["mu"]).compute_vel(F)
    direct = apply_kernel(f, c, NN @ F, w["eps"], w["mu"])
    print(f"matvec 4000/16000: {time.time() - t:.1f}s, nodes {tree.node_count}, "
          f"fmm vs direct {np.linalg.norm(vel - direct) / np.linalg.norm(direct):.2e}")
    d = dict(coarse=c, fine=f, F=F, eps=w["eps"], mu=w["mu"], cap=w["cap"], vel=vel, direct=direct)
    d.update(nn_arrays(NN))
    d.update(tree_arrays(tree))
    np.savez_compressed(os.path.join(OUT, "matvec_4000_16000.npz"), **d)


if __name__ == "__main__":
    which = sys.argv[1:] or ["sphere", "plain", "nearest", "split", "matvec"]
    if "sphere" in which:
        sphere_case()
    if "plain" in which:
        adaptive_plain_case()
    if "nearest" in which:
        adaptive_nearest_case()
    if "split" in which:
        split_case()
    if "matvec" in which:
        matvec_case()
