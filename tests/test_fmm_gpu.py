"""GPU parity of the KIFMM matvec (through the C ABI) against the FP64
oracle's per-node-LU restatement of the reference passes (golden fixtures
made by tests/golden/make_golden.py) and against dense direct sums.

Tolerances: FP64 mode reproduces the oracle to <= 1e-6 relative L2 on every
fixture (measured 1e-9 .. 4e-8).  Mixed mode (FP32 pair kernels, TF32 tensor-core M2L, FP64 check-to-equivalent
operators with Tikhonov regularization) must stay within 1e-4 of the FP64
direct sum and of the FP64 GPU result on well-posed inputs."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def tree_of(g):
    if "coarse" in g:
        NN = sp.csr_matrix((g["nn_data"], g["nn_indices"], g["nn_indptr"]))
        return nk.OcTree(g["coarse"], g["coarse"], nodeCapacity=int(g["cap"]), nearest=1, finePoints=g["fine"], NN=NN)
    if "src" in g:
        return nk.OcTree(g["src"], g["tgt"], nodeCapacity=int(g["cap"]))
    return nk.OcTree(g["points"], g["points"], nodeCapacity=int(g["cap"]))


FP64_TOL = {"sphere10_40": 1e-6, "adaptive_plain_1600": 1e-6, "adaptive_nearest_1200": 1e-6,
            "split_1500_700": 1e-6, "matvec_4000_16000": 1e-6}


@pytest.mark.parametrize("name", sorted(FP64_TOL))
def test_fp64_matches_oracle(name):
    g = load(name)
    t = tree_of(g)
    fmm = nk.KIFMM(t, [float(g["eps"]), float(g["mu"])])
    v = fmm.computeVel(g["F"])
    assert v.shape == g["vel"].shape
    e = rel(v, g["vel"])
    print(name, "fp64 vs oracle", e, "oracle vs direct", rel(g["vel"], g["direct"]))
    assert e <= FP64_TOL[name]


@pytest.mark.parametrize("name", sorted(FP64_TOL))
def test_near32_matches_fp64_and_oracle(name):
    """NEAR32: the reference's operator (exact check-to-equivalent inverses,
    every sum over equivalent densities in FP64) with the U-list P2P and the
    X-list P2L, whose sources are the forces, in FP32.  Their FP32 rounding
    reaches the velocities without passing an ill-conditioned inverse
    amplified, so the result stays within 1e-5 of FP64 mode and of the oracle
    on every fixture, the ill-posed NEAREST clouds included."""
    g = load(name)
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    v64 = nk.KIFMM(t, kp).computeVel(g["F"])
    fmm = nk.KIFMM(t, kp, precision="near32")
    fmm.autotune(1)
    v = fmm.computeVel(g["F"])
    print(name, "near32 vs fp64", rel(v, v64), "vs oracle", rel(v, g["vel"]))
    assert rel(v, v64) <= 1e-5 and rel(v, g["vel"]) <= 1e-5
    two = fmm.computeVel(np.stack([g["F"], -2.0 * g["F"]]), nrhs=2)
    assert np.array_equal(two[0], v) and rel(two[1], -2.0 * v) <= 1e-12


def test_near32_matches_fp64_at_scale():
    """The matvec-at-scale distribution at 60k force / 240k quadrature points
    (NEAREST sources outside their leaf boxes make the reference's exact
    check-to-equivalent solves ill-posed): NEAR32 within 1e-4 of FP64 mode,
    where the Tikhonov-regularized mixed mode is a different operator."""
    from nnkifmm.workloads import matvec_at_scale
    w = matvec_at_scale(60000, 240000)
    NN = nk.nearestMatrix(w["coarse"], w["fine"])
    t = nk.OcTree(w["coarse"], w["coarse"], nodeCapacity=64, nearest=1, finePoints=w["fine"], NN=NN)
    kp, F = [w["eps"], w["mu"]], w["forces"]
    v64 = nk.KIFMM(t, kp).computeVel(F)
    v = nk.KIFMM(t, kp, precision="near32").computeVel(F)
    vm = nk.KIFMM(t, kp, precision="mixed").computeVel(F)
    print("60k near32 vs fp64", rel(v, v64), "mixed vs fp64", rel(vm, v64))
    assert rel(v, v64) <= 1e-4


@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_plain_1600", "split_1500_700"])
def test_mixed_matches_fp64(name):
    g = load(name)
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    v64 = nk.KIFMM(t, kp).computeVel(g["F"])
    v32 = nk.KIFMM(t, kp, precision="mixed").computeVel(g["F"])
    e = rel(v32, v64)
    print(name, "mixed vs fp64", e, "mixed vs direct", rel(v32, g["direct"]))
    # The split fixture carries the reference's missing-P2L error (9% off the
    # direct sum), which makes the TF32 M2L rounding show at ~1e-4 there.
    assert e <= (2e-4 if name == "split_1500_700" else 1e-4)


def test_mixed_on_ill_posed_nearest_fixture():
    """NEAREST sources outside their leaf boxes make the exact check-to-
    equivalent solve ill-posed; the reference algorithm (and FP64 mode) is then
    ~1e-2 off the direct sum.  Mixed mode's regularized operators must be no
    worse than that against the direct sum."""
    g = load("adaptive_nearest_1200")
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    v64 = nk.KIFMM(t, kp).computeVel(g["F"])
    v32 = nk.KIFMM(t, kp, precision="mixed").computeVel(g["F"])
    print("fp64 vs direct", rel(v64, g["direct"]), "mixed vs direct", rel(v32, g["direct"]))
    assert rel(v32, g["direct"]) <= rel(v64, g["direct"])


@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_plain_1600"])
def test_mixed_vs_direct_sum(name):
    g = load(name)
    t = tree_of(g)
    v32 = nk.KIFMM(t, [float(g["eps"]), float(g["mu"])], precision="mixed").computeVel(g["F"])
    assert rel(v32, g["direct"]) <= 1e-4


@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_plain_1600"])
def test_generated_m2l_operators_match_streamed(name):
    """M2L operators generated inside the kernel give the streamed-image result."""
    g = load(name)
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    a = nk.KIFMM(t, kp, precision="mixed", m2l="images").computeVel(g["F"])
    b = nk.KIFMM(t, kp, precision="mixed", m2l="generate").computeVel(g["F"])
    assert rel(b, a) <= 1e-5


@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_plain_1600", "split_1500_700", "matvec_60k"])
def test_compressed_m2l_matches_full_operators(name):
    """The default tensor-core M2L on rank-256 compressed operators
    (B C_o B^T per level) against the full TF32 operator images and the FP32
    pair-kernel M2L: truncation and rounding stay at the full operators'
    TF32 rounding level."""
    if name == "matvec_60k":
        from nnkifmm.workloads import matvec_at_scale
        w = matvec_at_scale(60000, 240000)
        NN = nk.nearestMatrix(w["coarse"], w["fine"])
        t = nk.OcTree(w["coarse"], w["coarse"], nodeCapacity=64, nearest=1, finePoints=w["fine"], NN=NN)
        kp, F = [w["eps"], w["mu"]], w["forces"]
    else:
        g = load(name)
        t = tree_of(g)
        kp, F = [float(g["eps"]), float(g["mu"])], g["F"]
    comp = nk.KIFMM(t, kp, precision="mixed")
    assert comp.stats()["m2l_rank"] == 256
    a = comp.computeVel(F)
    b = nk.KIFMM(t, kp, precision="mixed", m2l="images").computeVel(F)
    c = nk.KIFMM(t, kp, precision="mixed", m2l="pairs").computeVel(F)
    print(name, "compressed vs pairs", rel(a, c), "full images vs pairs", rel(b, c))
    # both carry TF32 rounding of the operators (~1e-5 to 5e-5 on the well-posed
    # cases; the NEAREST cloud's ill-posed check-to-equivalent solves lift it)
    assert rel(a, c) <= max(1.5 * rel(b, c), 2e-5)
    if name in ("sphere10_40", "adaptive_plain_1600"):
        assert rel(a, c) <= 1e-4


@pytest.mark.parametrize("name", ["adaptive_nearest_1200", "matvec_4000_16000"])
def test_fp64_fourier_m2l_matches_fp64_pairs(name):
    """FP64 mode's Fourier-space M2L (FP64 spectra, the default) against its
    FP64 pair-kernel M2L: the same operator to rounding, amplified by the
    exact check-to-equivalent inverses (cond ~2e10)."""
    g = load(name)
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    a = nk.KIFMM(t, kp, m2l="pairs").computeVel(g["F"])
    b = nk.KIFMM(t, kp).computeVel(g["F"])
    print(name, "fp64 fourier vs fp64 pairs", rel(b, a), "vs oracle", rel(b, g["vel"]), rel(a, g["vel"]))
    assert rel(b, a) <= 1e-7


@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_nearest_1200", "matvec_4000_16000"])
def test_folded_m2m_l2l_matches_pair_sums(name):
    """Mixed mode (Tikhonov operators) with M2M and L2L folded into the
    check-to-equivalent products (nnk_fmm_set_fold) against the pair sums
    they replace: the same operator to the FP32 rounding of the replaced
    pair sums (the folded products run in FP64); measured 3e-7.  FP64 mode
    with the exact inverses refuses to fold (the folded products would lift
    FP64 rounding by cond ~1e10: 4e-5 on the NEAREST fixture)."""
    g = load(name)
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    fmm = nk.KIFMM(t, kp, precision="mixed")
    assert fmm.stats()["folded"] == 0  # off by default
    b = fmm.computeVel(g["F"])
    fmm.setFold(2)  # these trees are below the size where folding would pay
    folded = fmm.stats()["folded"]
    a = fmm.computeVel(g["F"])
    fmm.setFold(0)
    c = fmm.computeVel(g["F"])
    print(name, "mixed folded", folded, "folded vs pair sums", rel(a, b))
    assert np.array_equal(b, c)
    if name != "sphere10_40":  # the sphere's tree has no non-leaf node below the root
        assert folded == 1
    assert rel(a, b) <= 1e-6
    exact = nk.KIFMM(t, kp)
    exact.setFold(2)
    assert exact.stats()["folded"] == 0


C2E_TC_TOL = {"fp64": 1e-7, "near32": 1e-7, "mixed": 1e-5}


@pytest.mark.parametrize("precision", sorted(C2E_TC_TOL))
@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_nearest_1200", "split_1500_700", "matvec_4000_16000"])
def test_tensor_core_c2e_matches_fp64_simt(name, precision):
    """Check-to-equivalent products on the tensor cores (int8 digits, exact
    int32 sums combined in FP64) against the FP64 SIMT products:
    the same FP64 product to rounding, lifted by the exact inverses'
    condition number in FP64 mode (6e-9 to 1.3e-8, where FP64 mode is 1e-8
    to 6e-8 from the oracle with either); in mixed mode the 4 digits of a
    check column keep 28 bits below its largest entry and the 5 of an
    operator row 35, 1e-6 to 5e-6 from the SIMT product, within the mixed
    matvec's own 5e-5.  FP64 mode
    still matches the oracle."""
    g = load(name)
    t = tree_of(g)
    fmm = nk.KIFMM(t, [float(g["eps"]), float(g["mu"])], precision=precision)
    assert fmm.c2eMode() == 2  # the default: library DGEMM
    fmm.setC2E(1)
    assert fmm.c2eMode() == 1
    a = fmm.computeVel(g["F"])
    fmm.setC2E(0)
    assert fmm.c2eMode() == 0
    b = fmm.computeVel(g["F"])
    fmm.setC2E(1)
    c = fmm.computeVel(g["F"])
    print(name, precision, "tensor-core C2E vs SIMT", rel(a, b), "vs oracle", rel(a, g["vel"]), rel(b, g["vel"]))
    assert np.array_equal(a, c)
    # auto (-1): autotune keeps the faster form; the matvec is then that form's
    # (compared after autotune, which may also change the pair-kernel tiles)
    fmm.setC2E(-1)
    fmm.autotune()
    kept = fmm.c2eMode()
    d = fmm.computeVel(g["F"])
    fmm.setC2E(kept)
    assert np.array_equal(d, fmm.computeVel(g["F"]))
    assert rel(a, b) <= C2E_TC_TOL[precision]
    if precision == "fp64":
        assert rel(a, g["vel"]) <= FP64_TOL[name]


@pytest.mark.parametrize("precision", ["fp64", "near32", "mixed"])
@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_nearest_1200", "matvec_4000_16000"])
def test_library_dgemm_c2e_matches_simt(name, precision):
    """Check-to-equivalent products as one cuBLAS DGEMM per run of nodes
    sharing an operator (mode 2, the check vectors gathered and the products
    scattered) against the FP64 SIMT products: the same FP64 product summed
    in another order, lifted by the exact inverses' condition number (the
    tensor-core form's bound holds with room); FP64 mode still matches the
    oracle, and repeated calls give the same bits."""
    g = load(name)
    t = tree_of(g)
    fmm = nk.KIFMM(t, [float(g["eps"]), float(g["mu"])], precision=precision)
    assert fmm.c2eMode() == 2  # the default
    fmm.setC2E(0)
    b = fmm.computeVel(g["F"])
    fmm.setC2E(2)
    assert fmm.c2eMode() == 2
    a = fmm.computeVel(g["F"])
    assert np.array_equal(a, fmm.computeVel(g["F"]))
    fmm.setC2E(0)
    assert np.array_equal(b, fmm.computeVel(g["F"]))
    print(name, precision, "dgemm C2E vs SIMT", rel(a, b))
    assert rel(a, b) <= C2E_TC_TOL[precision]
    if precision == "fp64":
        assert rel(a, g["vel"]) <= FP64_TOL[name]


@pytest.mark.parametrize("precision", ["fp64", "near32", "mixed"])
@pytest.mark.parametrize("name", ["sphere10_40", "adaptive_nearest_1200", "split_1500_700", "matvec_4000_16000"])
def test_m2m_l2l_products_match_pair_sums(name, precision):
    """M2M and L2L as products with their kernel matrices (form 2, the
    default; form 1 for M2M alone) against the pair sums: the same check potentials to FP64 rounding,
    lifted by the check-to-equivalent inverses (the C2E forms' bound holds);
    FP64 mode still matches the oracle.  The statistics count the pairs the
    products take over (non-leaf nodes x 8 P^2 for each of M2M and L2L)."""
    g = load(name)
    t = tree_of(g)
    fmm = nk.KIFMM(t, [float(g["eps"]), float(g["mu"])], precision=precision)
    st = fmm.stats()
    a = fmm.computeVel(g["F"])  # the default, form 2: M2M and L2L products
    fmm.setM2MForm(1)  # M2M products, L2L pairs
    c = fmm.computeVel(g["F"])
    st1 = fmm.stats()
    fmm.setM2MForm(0)
    assert fmm.stats()["m2m_product_pairs"] == 0 and fmm.stats()["l2l_product_pairs"] == 0
    b = fmm.computeVel(g["F"])
    fmm.setM2MForm(2)
    assert np.array_equal(a, fmm.computeVel(g["F"]))
    par = np.asarray(t.nodeParents).ravel()
    lev = np.asarray(t.nodeLevel).ravel()
    # non-leaf nodes below the root (1-based parent ids, 0 = none); the root has no M2M of its own
    nonleaf = len({int(p) - 1 for p in par if p > 0 and lev[int(p) - 1] >= 1})
    pairs = nonleaf * 8 * st["surface_points"] ** 2
    assert st["m2m_product_pairs"] == pairs and st["l2l_product_pairs"] == pairs
    assert st1["m2m_product_pairs"] == pairs and st1["l2l_product_pairs"] == 0
    print(name, precision, "M2M/L2L products vs pair sums", rel(a, b), rel(c, b))
    assert rel(a, b) <= C2E_TC_TOL[precision] and rel(c, b) <= C2E_TC_TOL[precision]
    if precision == "fp64":
        assert rel(a, g["vel"]) <= FP64_TOL[name] and rel(c, g["vel"]) <= FP64_TOL[name]


@pytest.mark.parametrize("name", sorted(FP64_TOL))
def test_fourier_m2l_matches_pair_m2l(name):
    """The Fourier-space M2L (FP32 spectra) gives the FP32 pair-kernel M2L
    result."""
    g = load(name)
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    a = nk.KIFMM(t, kp, precision="mixed", m2l="pairs").computeVel(g["F"])
    b = nk.KIFMM(t, kp, precision="mixed", m2l="fft").computeVel(g["F"])
    assert rel(b, a) <= 1e-5


def test_sparse_matches_oracle():
    g = load("sphere10_40")
    fmm = nk.KIFMM(tree_of(g), [float(g["eps"]), float(g["mu"])])
    assert rel(fmm.computeVelSparse(g["F"]), g["vel_sparse"]) <= 1e-6


def test_reduced_matches_oracle():
    g = load("sphere10_40")
    fmm = nk.KIFMM(tree_of(g), [float(g["eps"]), float(g["mu"])])
    assert rel(fmm.reducedComputeVel(g["F"]), g["reduced"]) <= 1e-12
    assert rel(fmm.reducedSolve(g["U"]), g["reduced_solve"]) <= 1e-9


def test_layouts_and_multiple_rhs():
    g = load("adaptive_plain_1600")
    t = tree_of(g)
    kp = [float(g["eps"]), float(g["mu"])]
    F = g["F"]
    v = nk.KIFMM(t, kp).computeVel(F)
    v1 = nk.KIFMM(t, kp, GMRES=1, format=1).computeVel(F.ravel())
    v2 = nk.KIFMM(t, kp, GMRES=1, format=2).computeVel(F.T.ravel())
    assert np.array_equal(v1, v.ravel())
    assert np.array_equal(v2, v.T.ravel())
    two = nk.KIFMM(t, kp).computeVel(np.stack([F, 2 * F]), nrhs=2)
    assert np.array_equal(two[0], v) and rel(two[1], 2 * v) < 1e-14


def test_device_tensors_roundtrip():
    import torch
    g = load("sphere10_40")
    fmm = nk.KIFMM(tree_of(g), [float(g["eps"]), float(g["mu"])])
    Fd = torch.tensor(g["F"], device="cuda")
    vd = fmm.computeVel(Fd)
    assert vd.is_cuda
    assert np.array_equal(vd.cpu().numpy(), fmm.computeVel(g["F"]))


@pytest.mark.parametrize("precision", ["fp64", "near32", "mixed"])
def test_repeatable_bitwise(precision):
    """Every precision mode gives the same bits on every call: split pair
    tasks add their pieces in a fixed order, and the tensor-core M2L writes
    one partial block per work unit and adds a tile's blocks in unit order
    (no floating-point atomics)."""
    g = load("adaptive_nearest_1200")
    fmm = nk.KIFMM(tree_of(g), [float(g["eps"]), float(g["mu"])], precision=precision)
    a = fmm.computeVel(g["F"])
    for _ in range(3):
        assert np.array_equal(fmm.computeVel(g["F"]), a)


def test_linearity():
    g = load("adaptive_plain_1600")
    fmm = nk.KIFMM(tree_of(g), [float(g["eps"]), float(g["mu"])])
    rng = np.random.default_rng(0)
    A, B = rng.standard_normal(g["F"].shape), rng.standard_normal(g["F"].shape)
    lhs = fmm.computeVel(2.0 * A - 3.0 * B)
    rhs = 2.0 * fmm.computeVel(A) - 3.0 * fmm.computeVel(B)
    # the surface matrices have cond ~2e10, so FP64 rounding shows at ~1e-9
    assert rel(lhs, rhs) < 1e-8


def test_fmm_after_its_context_handle_is_destroyed():
    """Trees and FMMs hold their context: with the caller's context handle
    destroyed first, the FMM still evaluates (the same result) and the
    handles can be destroyed afterwards."""
    import ctypes
    L = nk._lib
    g = np.load(os.path.join(GOLDEN, "sphere10_40.npz"))
    x = np.ascontiguousarray(g["coarse"])
    n, kp = len(x), [float(g["eps"]), float(g["mu"])]
    ref = nk.KIFMM(nk.OcTree(x, x, nodeCapacity=int(g["cap"])), kp)
    f = np.ascontiguousarray(np.random.default_rng(4).standard_normal(3 * n))
    ctx, tree, fmm = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    assert L.lib.nnk_ctx_create(0, ctypes.byref(ctx)) == L.NNK_OK
    tp = L.TreeParams(int(g["cap"]), 20, 0, 0)
    assert L.lib.nnk_tree_build(ctx, L.ptr(x), n, L.ptr(x), n, None, 0, None, None, None, ctypes.byref(tp),
                                ctypes.byref(tree)) == L.NNK_OK
    fp = L.FmmParams(kp[0], kp[1], 6, 1, L.PREC_FP64, 0, 0.0)
    assert L.lib.nnk_fmm_create(ctx, tree, ctypes.byref(fp), ctypes.byref(fmm)) == L.NNK_OK
    assert L.lib.nnk_ctx_destroy(ctx) == L.NNK_OK
    out = np.empty(3 * n)
    assert L.lib.nnk_fmm_apply(fmm, L.ptr(f), L.ptr(out), 1, 1, 0) == L.NNK_OK  # layout rows, host buffers
    assert np.array_equal(out, ref.computeVel(f).ravel())
    assert L.lib.nnk_fmm_destroy(fmm) == L.NNK_OK
    assert L.lib.nnk_tree_destroy(tree) == L.NNK_OK


@pytest.mark.parametrize("name", ["adaptive_nearest_1200", "matvec_4000_16000"])
def test_fourier_m2l_family_statistics(name):
    """The parent-grouped Fourier M2L's record and group counts (the L2
    traffic of its accumulation) against a count from the exported tree: a
    record per (parent of a V-list target, parent of its V-list source), a
    group per record and child difference (pos_v - pos_i, both child positions
    in their parents)."""
    g = load(name)
    t = tree_of(g)
    st = nk.KIFMM(t, [float(g["eps"]), float(g["mu"])]).stats()
    par = np.asarray(t.nodeParents).ravel().astype(np.int64) - 1  # 1-based ids, 0 = none
    cor = np.asarray(t.nodeCorners)
    root = int(np.where(par < 0)[0][0])
    wid = cor[:, 3] - cor[:, 0]
    ijk = np.rint((cor[:, :3] - cor[root, :3]) / wid[:, None]).astype(np.int64)
    off, ids = t.interaction_list(1)
    ids = ids.astype(np.int64) - 1
    records, groups = set(), set()
    for i in range(len(par)):
        for v in ids[off[i]:off[i + 1]]:
            P, N = int(par[i]), int(par[v])
            e = tuple(int(x) for x in (ijk[v] - 2 * ijk[N]) - (ijk[i] - 2 * ijk[P]))
            records.add((P, N))
            groups.add((P, N, e))
    assert st["m2l_family"] == 1 and st["m2l_frequencies"] == 11 * 11 * 6
    assert st["m2l_records"] == len(records) and st["m2l_groups"] == len(groups)
    assert st["m2l_pairs"] == int(off[-1])


def test_measure_l2_read():
    """The L2 read rate used as the Fourier accumulation's second roofline:
    a streaming read of an L2-resident buffer runs well above the HBM rate."""
    gbs = nk.context(0).measure_l2_read()
    print("L2 read", gbs, "GB/s")
    assert 8000.0 < gbs < 40000.0
