"""The GPU builders of the octree's node structure and of the nearest-
neighbour matrix against the host builders (which are bit-exact against the
oracle, tests/test_tree_cpu.py): every exported array identical."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN
from nnkifmm.workloads import cube_sphere, matvec_at_scale, prolate_spheroid

pytestmark = pytest.mark.gpu


def exported(t):
    out = dict(nodes=t.nodeCount, level=t.nodeLevel, parent=t.nodeParents, children=t.nodeChildren,
               corners=t.nodeCorners, point_index=t.pointIndex)
    for k, name in enumerate("UVWX"):
        off, ids = t.interaction_list(k)
        out["off" + name], out["ids" + name] = off, ids
    return out


def same(a, b):
    assert a["nodes"] == b["nodes"]
    for k in a:
        if k != "nodes":
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def cases():
    out = []
    for name in ["sphere10_40", "adaptive_nearest_1200", "adaptive_plain_1600", "split_1500_700"]:
        g = np.load(os.path.join(GOLDEN, name + ".npz"))
        if "coarse" in g:
            NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
            out.append((name, dict(potPoints=g["coarse"], targetPoints=g["coarse"], nodeCapacity=int(g["cap"]),
                                   nearest=1, finePoints=g["fine"], NN=NN)))
        elif "src" in g:
            out.append((name, dict(potPoints=g["src"], targetPoints=g["tgt"], nodeCapacity=int(g["cap"]))))
        else:
            out.append((name, dict(potPoints=g["points"], targetPoints=g["points"], nodeCapacity=int(g["cap"]))))
    w = matvec_at_scale(60000, 240000)
    out.append(("matvec_60k", dict(potPoints=w["coarse"], targetPoints=w["coarse"], nodeCapacity=64)))
    X = prolate_spheroid(0.6, 2.0, 0.03)
    out.append(("prolate", dict(potPoints=X, targetPoints=X, nodeCapacity=200)))
    return out


@pytest.mark.parametrize("name,kw", cases(), ids=[c[0] for c in cases()])
def test_gpu_tree_matches_host(name, kw):
    same(exported(nk.OcTree(builder="gpu", **kw)), exported(nk.OcTree(builder="host", **kw)))


def test_gpu_tree_max_depth_error():
    x = np.random.default_rng(3).random((500, 3))
    with pytest.raises(nk.MaxDepthError):
        nk.OcTree(x, x, nodeCapacity=1, maxDepth=4, builder="gpu")
    with pytest.raises(nk.MaxDepthError):
        nk.OcTree(x, x, nodeCapacity=1, maxDepth=4, builder="host")


@pytest.mark.parametrize("case", ["sphere", "prolate", "cloud", "lattice_ties"])
def test_gpu_nearest_matrix_matches_host(case):
    rng = np.random.default_rng(11)
    if case == "sphere":
        c, f = cube_sphere(1.0, (0, 0, 0), 12), cube_sphere(1.0, (0, 0, 0), 48)
    elif case == "prolate":
        c, f = prolate_spheroid(0.7, 2.1, 0.05), prolate_spheroid(0.7, 2.1, 0.0125)
    elif case == "cloud":
        w = matvec_at_scale(40000, 160000)
        c, f = w["coarse"], w["fine"]
    else:  # exact ties: a lattice of coarse points and fine points between them
        g = np.arange(8, dtype=float)
        c = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
        f = np.concatenate([c + 0.5, c + np.array([0.5, 0.0, 0.0]), rng.random((500, 3)) * 7])
    a = nk.nearestMatrix(c, f)
    b = nk.nearestMatrix(c, f, builder="host")
    assert np.array_equal(a.indptr, b.indptr)
    assert np.array_equal(a.indices, b.indices)
    assert np.array_equal(a.data, b.data)
    if case == "lattice_ties":
        assert np.diff(a.indptr).max() == 8  # the cube centres: 8 nearest corners, weight 1/8


def test_gpu_tree_lists_and_nn_match_oracle_4000_16000():
    """Tree, lists and NN built on the GPU (NN searched on the device, nodes
    partitioned on the device) for the matvec-at-scale distribution at 4000 /
    16000 points, against the oracle's fixture directly, bit for bit."""
    g = np.load(os.path.join(GOLDEN, "matvec_4000_16000.npz"))
    NN = nk.nearestMatrix(g["coarse"], g["fine"])
    A = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]), shape=NN.shape)
    assert (A != NN).nnz == 0 and A.nnz == NN.nnz
    t = nk.OcTree(g["coarse"], g["coarse"], nodeCapacity=int(g["cap"]), nearest=1, finePoints=g["fine"])
    assert (t.NN != A).nnz == 0
    assert np.array_equal(t.nodeLevel, g["level"]) and np.array_equal(t.nodeParents, g["parent"])
    assert np.array_equal(t.nodeChildren, g["children"]) and np.array_equal(t.nodeCorners, g["corners"])
    assert np.array_equal(t.pointIndex, g["point_index"])
    for k, name in enumerate("UVWX"):
        off, ids = t.interaction_list(k)
        assert np.array_equal(off, g[f"list_{name}_off"]) and np.array_equal(ids, g[f"list_{name}_ids"]), name
