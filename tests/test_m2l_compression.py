"""The mathematics behind the compressed tensor-core M2L, checked on the CPU
with the oracle's kernel and surfaces: the translation operators satisfy
T_o^T = T_{-o} (so one basis serves both sides), and the rank-256 basis of
sum_o T_o T_o^T over the 316 far offsets, rotated by a normalized Hadamard
matrix, reproduces the summed M2L of a physical equivalent density to ~1e-6."""
import numpy as np
from scipy.linalg import hadamard

from oracle.kernel import kernel
from oracle.surfaces import upsurf


def far_offsets():
    return [(x, y, z) for x in range(-3, 4) for y in range(-3, 4) for z in range(-3, 4)
            if max(abs(x), abs(y), abs(z)) >= 2]


def operators(w, eps):
    tgt = upsurf([0, 0, 0, w, w, w])
    out = {}
    for o in far_offsets():
        src = upsurf([o[0] * w, o[1] * w, o[2] * w, (o[0] + 1) * w, (o[1] + 1) * w, (o[2] + 1) * w])
        out[o] = kernel(src, tgt, eps, 1.0)  # source density at offset o -> target check surface
    return out


def test_transpose_is_the_opposite_offset():
    T = operators(0.25, 0.01)
    assert len(T) == 316
    for o in [(2, 0, 0), (3, -2, 1), (-3, 3, 3)]:
        mo = tuple(-c for c in o)
        assert np.abs(T[o].T - T[mo]).max() <= 1e-14 * np.abs(T[o]).max()


def test_rank_256_rotated_basis_reproduces_the_summed_m2l():
    w, eps = 1.0 / 64, 1e-3
    T = operators(w, eps)
    G = sum(t @ t.T for t in T.values())
    _, U = np.linalg.eigh(G)
    B = U[:, -256:] @ (hadamard(256) / 16.0)
    assert np.allclose(B.T @ B, np.eye(256), atol=1e-12)
    # an equivalent density of sources inside the box (least squares on the 3x check surface)
    rng = np.random.default_rng(1)
    xs, fs = rng.random((200, 3)) * w, rng.standard_normal((200, 3))
    chk = upsurf([-w, -w, -w, 2 * w, 2 * w, 2 * w])
    u = np.linalg.lstsq(kernel(upsurf([0, 0, 0, w, w, w]), chk, eps, 1.0),
                        kernel(xs, chk, eps, 1.0) @ fs.ravel(), rcond=1e-10)[0]
    exact = sum(t @ u for t in T.values())
    comp = B @ sum((B.T @ t @ B) @ (B.T @ u) for t in T.values())
    assert np.linalg.norm(comp - exact) <= 1e-5 * np.linalg.norm(exact)
