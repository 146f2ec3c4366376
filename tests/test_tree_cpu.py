"""Bit-exact parity of the library's octree, U/V/W/X lists and NN matrix
(through the C ABI, host part; no GPU needed) with the oracle restatement of
Classes/OcTree.m and Tools/Nearest/nearestMatrix.m."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN, ROOT
from oracle.geometry import sphere
from oracle.nearest import nearest_matrix
from oracle.octree import OcTree as OracleTree


def assert_same_tree(a, b):
    assert a.node_count == b.nodeCount
    assert np.array_equal(a.level[1:], b.nodeLevel)
    assert np.array_equal(a.parent[1:], b.nodeParents)
    assert np.array_equal(a.children[1:], b.nodeChildren)
    assert np.array_equal(a.corners[1:], b.nodeCorners)  # bit-exact FP64 midpoints
    assert np.array_equal(a.point_index, b.pointIndex)
    assert np.array_equal(a.potentials, b.potentials) and np.array_equal(a.targets, b.targets)
    inter = b.interactions
    for i in range(1, a.node_count + 1):
        for k, lst in enumerate([a.U, a.V, a.W, a.X]):
            assert np.array_equal(lst[i], inter[i - 1][k]), (i, "UVWX"[k], lst[i], inter[i - 1][k])


def mixed(rng, n):
    u = rng.random((n // 2, 3))
    cen = rng.uniform(0.2, 0.8, (3, 3))
    rad = rng.uniform(0.05, 0.2, 3)
    d = rng.standard_normal((n - n // 2, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    k = rng.integers(0, 3, n - n // 2)
    return np.concatenate([u, cen[k] + rad[k, None] * d])


@pytest.mark.parametrize("seed,n,cap", [(0, 1500, 64), (1, 1500, 20), (2, 900, 8), (3, 3000, 50)])
def test_tree_and_lists_match_oracle(seed, n, cap):
    x = mixed(np.random.default_rng(seed), n)
    assert_same_tree(OracleTree(x, x, node_capacity=cap), nk.OcTree(x, x, nodeCapacity=cap))


def test_tree_clustered_deep():
    rng = np.random.default_rng(7)
    z = np.concatenate([rng.normal(0.3, 0.005, (1000, 3)), rng.random((300, 3))])
    assert_same_tree(OracleTree(z, z, node_capacity=12), nk.OcTree(z, z, nodeCapacity=12))


def test_tree_split_sources_targets():
    rng = np.random.default_rng(8)
    s = mixed(rng, 1200)
    t = np.concatenate([rng.random((400, 3)) * 0.6, s[:50]])  # some targets coincide with sources
    assert_same_tree(OracleTree(s, t, node_capacity=25), nk.OcTree(s, t, nodeCapacity=25))


def test_tree_sphere_488_points():
    c = sphere(1.0, [0, 0, 0], 10)
    assert_same_tree(OracleTree(c, c, node_capacity=60), nk.OcTree(c, c, nodeCapacity=60))


@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_plain_1600", "adaptive_nearest_1200", "split_1500_700",
                                  "matvec_4000_16000"])
def test_tree_matches_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    if "coarse" in g:
        NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
        t = nk.OcTree(g["coarse"], g["coarse"], nodeCapacity=int(g["cap"]), nearest=1, finePoints=g["fine"], NN=NN)
    elif "src" in g:
        t = nk.OcTree(g["src"], g["tgt"], nodeCapacity=int(g["cap"]))
    else:
        t = nk.OcTree(g["points"], g["points"], nodeCapacity=int(g["cap"]))
    assert np.array_equal(t.nodeLevel, g["level"])
    assert np.array_equal(t.nodeParents, g["parent"])
    assert np.array_equal(t.nodeChildren, g["children"])
    assert np.array_equal(t.nodeCorners, g["corners"])
    assert np.array_equal(t.pointIndex, g["point_index"])
    for k, name_ in enumerate("UVWX"):
        off, ids = t.interaction_list(k)
        assert np.array_equal(off, g[f"list_{name_}_off"]) and np.array_equal(ids, g[f"list_{name_}_ids"])


def test_nearest_matrix_matches_oracle():
    rng = np.random.default_rng(11)
    c = mixed(rng, 2000)
    f = np.concatenate([rng.random((3000, 3)), c[:100] + 1e-3, rng.random((50, 3)) * 3 - 1])  # some outside
    A, B = nearest_matrix(c, f), nk.nearestMatrix(c, f)
    assert (A != B).nnz == 0 and A.nnz == B.nnz


def test_nearest_matrix_exact_ties():
    g = np.array([[i, j, k] for i in range(6) for j in range(6) for k in range(6)], float) * 0.1
    f = np.concatenate([g[:-1] + 0.05, g + [0.05, 0, 0], g])
    A, B = nearest_matrix(g, f), nk.nearestMatrix(g, f)
    assert (A != B).nnz == 0
    assert B.getnnz(axis=1).max() == 8  # cell centres tie with 8 corners


def test_sphere_nearest_matches_oracle():
    c, f = sphere(1.0, [0, 0, 0], 10), sphere(1.0, [0, 0, 0], 40)
    assert (nearest_matrix(c, f) != nk.nearestMatrix(c, f)).nnz == 0


def test_max_depth_error_message():
    x = np.array([[0, 0, 0], [1e-9, 0, 0], [1, 1, 1]], float)
    with pytest.raises(nk.MaxDepthError, match="Max level reached: Increase Max Depth"):
        nk.OcTree(x, x, nodeCapacity=1, maxDepth=8)


def test_capacity_clamped_to_points_minus_one():
    x = np.random.default_rng(0).random((10, 3))
    t = nk.OcTree(x, x, nodeCapacity=200)
    assert t.nodeCapacity == 9 and t.nodeCount >= 9  # root always divides (OcTree.m:105)


def test_bad_inputs_rejected():
    x = np.random.default_rng(0).random((10, 3))
    with pytest.raises(nk.NNKError):
        nk.OcTree(np.vstack([x, x[:1]]), np.vstack([x, x[:1]]))  # duplicate potential rows
    y = x.copy()
    y[3, 1] = np.nan
    with pytest.raises(nk.NNKError):
        nk.OcTree(y, y)
    with pytest.raises(nk.NNKError):  # NEAREST needs targets == potentials
        nk.OcTree(x, x[:5], nearest=1, finePoints=x)


_TREE_ARRAYS = """
import sys, numpy as np, scipy.sparse as sp
import nnkifmm as nk
x = np.load(sys.argv[1]); f = np.load(sys.argv[2])
NN = nk.nearestMatrix(x, f, builder="host")
t = nk.OcTree(x, x, nodeCapacity=8, nearest=1, finePoints=f, NN=NN, builder="host")
out = dict(level=t.nodeLevel, parent=t.nodeParents, children=t.nodeChildren, corners=t.nodeCorners,
           point_index=t.pointIndex, nn_indptr=NN.indptr, nn_indices=NN.indices, nn_data=NN.data)
for k in range(4):
    out[f"off{k}"], out[f"ids{k}"] = t.interaction_list(k)
np.savez(sys.argv[3], **out)
"""


def test_large_tree_independent_of_thread_count(tmp_path):
    """Above a few thousand nodes (or 65,536 points) the host builder checks
    the points for duplicates, builds the U/V/W lists and sorts the NN rows on
    OpenMP threads; a process held to one thread gives the same arrays."""
    import subprocess
    import sys
    rng = np.random.default_rng(21)
    x = mixed(rng, 120_000)
    f = np.concatenate([mixed(rng, 150_000), x[:2000] + 1e-4])
    np.save(tmp_path / "x.npy", x)
    np.save(tmp_path / "f.npy", f)
    script = tmp_path / "arrays.py"
    script.write_text(_TREE_ARRAYS)
    runs = {}
    for threads in ("1", "4"):
        path = os.pathsep.join([ROOT, os.path.join(ROOT, "stokes-nnkifmm_b200"), os.environ.get("PYTHONPATH", "")])
        env = dict(os.environ, OMP_NUM_THREADS=threads, PYTHONPATH=path)
        out = tmp_path / f"t{threads}.npz"
        subprocess.run([sys.executable, str(script), str(tmp_path / "x.npy"), str(tmp_path / "f.npy"), str(out)],
                       check=True, env=env, timeout=600)
        runs[threads] = np.load(out)
    a, b = runs["1"], runs["4"]
    assert a["level"].size > 2048
    for k in a.files:
        assert np.array_equal(a[k], b[k]), k


def test_large_duplicate_rows_rejected():
    """The duplicate check of potPoints on many threads: a repeated row, and a
    row equal to another up to the sign of zero (rows compare by value)."""
    x = np.random.default_rng(22).random((100_000, 3))
    x[500] = [0.0, 0.25, 0.75]
    for extra in (x[77:78], np.array([[-0.0, 0.25, 0.75]])):
        y = np.concatenate([x[:60_000], extra, x[60_000:]])
        with pytest.raises(nk.NNKError, match="duplicate"):
            nk.OcTree(y, y, nodeCapacity=64, builder="host")


def _lattice(n):
    g = np.arange(n) / (n - 1.0)
    return np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)


@pytest.mark.parametrize("case", ["on_split_planes", "planar", "line", "two_scales", "negative_zero"])
def test_tree_degenerate_inputs_match_oracle(case):
    """Inputs where the reference's rules decide: points exactly on the
    midpoint planes (strict p > centre), a flat and a one-dimensional cloud,
    two clusters five decades apart, and -0.0 coordinates."""
    rng = np.random.default_rng(31)
    if case == "on_split_planes":
        x, cap = _lattice(9), 20  # 729 points, every dyadic midpoint is a lattice plane
    elif case == "planar":
        x = rng.random((1500, 3))
        x[:, 2] = 0.25
        cap = 30
    elif case == "line":
        x = np.zeros((800, 3))
        x[:, 0] = np.sort(rng.random(800))
        x[:, 1] = 0.5
        cap = 16
    elif case == "two_scales":
        x = np.concatenate([rng.random((600, 3)), 0.3 + 1e-5 * rng.random((300, 3))])
        cap = 40
    else:
        x = rng.random((900, 3)) - 0.5
        x[:40, 1] = -0.0
        x[40:80, 1] = 0.0
        x[40:80, 0] += 1e-3  # distinct rows, equal coordinates of either sign
        cap = 25
    depth = 23 if case == "two_scales" else 21  # 23: the library's largest maxDepth
    t = nk.OcTree(x, x, nodeCapacity=cap, maxDepth=depth)
    assert_same_tree(OracleTree(x, x, node_capacity=cap, max_depth=depth), t)
    if case == "two_scales":
        assert t.nodeLevel.max() >= 17


def test_nearest_matrix_coincident_and_planar_ties():
    """Fine points on coarse points (distance 0), on edge midpoints of a flat
    lattice (2-way ties) and on its cell centres (4-way ties), bit for bit
    against the oracle, host and default builders."""
    g = np.arange(7) / 6.0
    c = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    c = np.concatenate([c, np.full((len(c), 1), 0.5)], axis=1)
    h = 0.5 / 6.0
    f = np.concatenate([c, c[:-1] + [h, 0, 0], c[:30] + [h, h, 0], c[5:25] + [0, 0, 0.3]])
    A = nearest_matrix(c, f)
    for builder in ("host", "auto"):
        B = nk.nearestMatrix(c, f, builder=builder)
        assert (A != B).nnz == 0 and A.nnz == B.nnz
    assert B.getnnz(axis=1).max() == 4 and np.all(B[:len(c)].getnnz(axis=1) == 1)


@pytest.mark.parametrize("case,code,message", [
    ("nan_potential", 3, "non-finite potential point"),
    ("inf_target", 3, "non-finite target point"),
    ("inf_fine", 3, "non-finite fine point"),
    ("no_points", 1, "no points"),
    ("max_depth_above_23", 1, "maxDepth above 23"),
])
def test_host_fault_injection(case, code, message):
    """Bad inputs come back as status codes with the reference's or a plain
    message, before any device work (host builder)."""
    rng = np.random.default_rng(51)
    x = rng.random((60, 3))
    t = rng.random((30, 3))
    f = rng.random((90, 3))
    kw = dict(nodeCapacity=10, builder="host")
    if case == "nan_potential":
        x[7, 2] = np.nan
        args = (x, t)
    elif case == "inf_target":
        t[3, 0] = np.inf
        args = (x, t)
    elif case == "inf_fine":
        f[11, 1] = -np.inf
        args, kw = (x, x), dict(kw, nearest=1, finePoints=f, NN=nk.nearestMatrix(x, rng.random((90, 3)), builder="host"))
    elif case == "no_points":
        args = (np.zeros((0, 3)), np.zeros((0, 3)))
    else:
        args, kw = (x, x), dict(kw, maxDepth=24)
    with pytest.raises(nk.NNKError, match=message) as e:
        nk.OcTree(*args, **kw)
    assert e.value.code == code


def test_nearest_without_fine_points_rejected():
    x = np.random.default_rng(52).random((40, 3))
    with pytest.raises(ValueError, match="finePoints"):  # the host mirror, before the C ABI
        nk.OcTree(x, x, nodeCapacity=10, nearest=1, builder="host")


def test_nearest_matrix_matches_golden_4000_16000():
    """NN of the matvec-at-scale distribution at 4000 / 16000 points (host
    builder) against the oracle's fixture, bit for bit."""
    g = np.load(os.path.join(GOLDEN, "matvec_4000_16000.npz"))
    A = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]), shape=(len(g["fine"]), len(g["coarse"])))
    B = nk.nearestMatrix(g["coarse"], g["fine"], builder="host")
    assert (A != B).nnz == 0 and A.nnz == B.nnz
