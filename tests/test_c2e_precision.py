"""Why the check-to-equivalent product stays FP64 in mixed precision, checked
on the CPU with the oracle's kernel and surfaces.  For a leaf-sized box
(eps = 1e-3, p = 6, Tikhonov operator lam = 1e-5 sigma_max, cond(K) ~ 2e10),
the far field of the upward equivalent density, at V-list distances, against
the direct sum of the box's sources:
  * FP64 operator and FP64 accumulation, on an FP32 check potential (the GPU's
    mixed mode): the FP64 error, ~1e-5;
  * FP32 accumulation, even of an exact (two-float) operator: ~1e-4 and above,
    the mixed mode's whole error budget;
  * one TF32 product: above 1e-2.
So a tensor-core form of this product needs exact accumulation, not TF32
terms accumulated in FP32: int8 slices of the operator (5, one exponent per
row) and of the check potentials (4, one exponent per column), multiplied with
exact integer sums and combined in FP64 (the Ozaki scheme), give the FP64
product's error with 14 slice products."""
import numpy as np
import pytest

from oracle.kernel import apply_kernel, kernel
from oracle.surfaces import downsurf, upsurf


def tf32(a):
    """Round to TF32 (10 explicit mantissa bits), nearest, ties away."""
    x = np.asarray(a, np.float32).copy()
    u = x.view(np.uint32)
    u += np.uint32(0x1000)
    u &= np.uint32(0xFFFFE000)
    return x


def setup(w, seed):
    rng = np.random.default_rng(seed)
    eps = 1e-3
    lo = np.array([0.3, 0.4, 0.5])
    box = np.concatenate([lo, lo + w])
    us, ds = upsurf(box), downsurf(box)
    K = kernel(us, ds, eps, 1.0)
    lam = 1e-5 * np.linalg.norm(K, 2)
    A = np.linalg.solve(K.T @ K + lam ** 2 * np.eye(K.shape[1]), K.T)
    src = lo + w * rng.random((300, 3))
    f = rng.standard_normal((300, 3))
    check = apply_kernel(src, ds, f, eps, 1.0).reshape(-1)
    d = rng.standard_normal((400, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tgt = lo + w / 2 + d * w * rng.uniform(2.5, 3.5, (400, 1))
    direct = apply_kernel(src, tgt, f, eps, 1.0).reshape(-1)

    def err(e):
        u = apply_kernel(us, tgt, np.asarray(e, np.float64).reshape(-1, 3), eps, 1.0).reshape(-1)
        return np.linalg.norm(u - direct) / np.linalg.norm(direct)
    return A, check, err


@pytest.mark.parametrize("w", [1 / 8, 1 / 32])
def test_c2e_needs_fp64_accumulation(w):
    A, check, err = setup(w, 1)
    c32 = check.astype(np.float32)
    e64 = err(A @ check)
    assert e64 < 3e-5
    assert err(A @ c32.astype(np.float64)) < 1.2 * e64           # FP32 check, FP64 operator and sums
    Ah = A.astype(np.float32)
    Al = (A - Ah).astype(np.float32)
    assert err(Ah @ c32 + Al @ c32) > 3 * e64                      # exact operator, FP32 sums
    assert err(Ah @ c32) > 5 * e64                                 # FP32 operator
    assert err(tf32(A).astype(np.float64) @ tf32(c32).astype(np.float64)) > 1e-2  # one TF32 product


def int8_slices(X, k, axis):
    """k int8 slices of X, X ~ 2^e * sum_t D_t 128^-(t+1), one power-of-two
    exponent e per row (axis=1) or per column (axis=0) (the Ozaki scheme)."""
    m = np.abs(X).max(axis=axis, keepdims=True)
    e = np.ceil(np.log2(np.where(m > 0, m, 1.0)))
    r = X / 2.0 ** e
    D = []
    for _ in range(k):
        r = r * 128.0
        d = np.clip(np.rint(r), -127, 127)
        r = r - d
        D.append(d.astype(np.int64))
    return D, e


@pytest.mark.parametrize("w", [1 / 8, 1 / 32, 1 / 128])
def test_int8_slice_product_keeps_the_fp64_accuracy(w):
    """5 operator slices x 4 check slices, the 14 products with t + u <= 4,
    each an exact integer sum (|sum| < 2^31: 456 x 127^2 x 4 products of one
    scale), combined in FP64: the far-field error of the FP64 product."""
    A, check, err = setup(w, 1)
    c = check.astype(np.float32).astype(np.float64).reshape(-1, 1)
    DA, ea = int8_slices(A, 5, 1)
    DC, ec = int8_slices(c, 4, 0)
    acc = {}
    for t in range(5):
        for u in range(4):
            if t + u <= 4:
                acc[t + u] = acc.get(t + u, 0) + DA[t] @ DC[u]
    assert max(np.abs(v).max() for v in acc.values()) < 2 ** 31
    e = sum(acc[s].astype(np.float64) * 2.0 ** (-7 * (s + 2)) for s in sorted(acc, reverse=True))
    e = (e * 2.0 ** ea * 2.0 ** ec).ravel()
    e64 = err(A @ c.ravel())
    assert err(e) < 1.05 * e64


def truncation_digits(X, k, axis):
    """The digits of the tensor-core C2E (csrc/c2e_tc.cu): exponent e with
    |x| / 2^e < 1 over the row (axis=1) or column (axis=0), then k digits by
    truncation toward zero, so every digit is in [-127, 127] and every step is
    exact in FP64."""
    m = np.abs(X).max(axis=axis, keepdims=True)
    e = np.where(m > 0, np.floor(np.log2(np.where(m > 0, m, 1.0))) + 1, 0.0)
    r = X / 2.0 ** e
    D = []
    for _ in range(k):
        r = r * 128.0
        d = np.trunc(r)
        r = r - d
        D.append(d.astype(np.int64))
    return D, e


@pytest.mark.parametrize("w", [1 / 16, 1 / 64])
def test_nine_digit_product_matches_fp64_on_the_exact_inverse(w):
    """FP64 mode: the exact inverse (cond ~1e10) on a NEAREST-like check
    (sources up to 0.3 widths outside the box), whose rows cancel by ~1e5.
    9 x 9 digits, levels t + u < 9 (45 products, each level an exact int32
    sum), against the product in extended precision: 5e-13, ten times closer
    than the FP64 product itself (6e-12: its sums round, the digit sums do
    not); 8 x 8 digits: 6e-11."""
    rng = np.random.default_rng(1)
    eps = 1e-3
    lo = np.array([0.3, 0.4, 0.5])
    box = np.concatenate([lo, lo + w])
    us, ds = upsurf(box), downsurf(box)
    A = np.linalg.inv(kernel(us, ds, eps, 1.0))
    src = lo - 0.3 * w + 1.6 * w * rng.random((300, 3))
    f = rng.standard_normal((300, 3))
    c = apply_kernel(src, ds, f, eps, 1.0).reshape(-1, 1)
    ref = (A.astype(np.longdouble) @ c.astype(np.longdouble)).astype(np.float64).ravel()
    fp64 = np.linalg.norm((A @ c).ravel() - ref) / np.linalg.norm(ref)
    errs = {}
    for s_ in (8, 9):
        DA, ea = truncation_digits(A, s_, 1)
        DC, ec = truncation_digits(c, s_, 0)
        lev = {}
        for t in range(s_):
            for u in range(s_ - t):
                lev[t + u] = lev.get(t + u, 0) + DA[t] @ DC[u]
        assert max(np.abs(v).max() for v in lev.values()) < 2 ** 31
        out = sum(lev[l].astype(np.float64) * 2.0 ** (-7 * (l + 2)) for l in sorted(lev, reverse=True))
        out = (out * 2.0 ** ea * 2.0 ** ec).ravel()
        errs[s_] = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert errs[9] <= 2 * max(fp64, 1e-13)
    assert errs[8] > errs[9]
