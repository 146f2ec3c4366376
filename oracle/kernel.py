"""Regularized Stokeslet kernel and its block products (FP64).

Test infrastructure only (see oracle/__init__.py).
"""
import numpy as np


def kernel(x, x0, eps, mu):
    """Dense Stokeslet matrix S (3M x 3N) between sources ``x`` (N,3) and
    targets ``x0`` (M,3); Tools/kernel.m:15-49.

    r = x0 - x (target minus source, kernel.m:23-25),
    S_ij = (r_i r_j + delta_ij (r^2 + 2 eps^2)) / (8 pi mu (r^2+eps^2)^{3/2}),
    rows/cols interleaved [x1 y1 z1 x2 ...] (kernel.m:36-47).
    """
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    x0 = np.asarray(x0, dtype=np.float64).reshape(-1, 3)
    M, N = x0.shape[0], x.shape[0]
    rx = x0[:, 0:1] - x[:, 0][None, :]
    ry = x0[:, 1:2] - x[:, 1][None, :]
    rz = x0[:, 2:3] - x[:, 2][None, :]
    r2 = rx * rx + ry * ry + rz * rz
    invs = (1.0 / ((r2 + eps ** 2) ** 1.5)) * (1.0 / (8.0 * np.pi * mu))
    S = np.zeros((3 * M, 3 * N))
    comps = (rx, ry, rz)
    iso = r2 + 2.0 * eps ** 2
    for a in range(3):
        for b in range(3):
            blk = comps[a] * comps[b]
            if a == b:
                blk = blk + iso
            S[a::3, b::3] = blk * invs
    return S


def apply_kernel(x, x0, f, eps, mu, block=4096):
    """u(x0) = S(x -> x0) f without forming the whole matrix at once;
    the blocked product of Tools/Other/blockcomputation.m:17-29.

    ``f`` is (N,3); returns (M,3).
    """
    x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
    x0 = np.asarray(x0, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(f, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((x0.shape[0], 3))
    if x.shape[0] == 0 or x0.shape[0] == 0:
        return out
    c = 1.0 / (8.0 * np.pi * mu)
    e2 = eps * eps
    for s in range(0, x0.shape[0], block):
        t = x0[s:s + block]
        r = t[:, None, :] - x[None, :, :]
        r2 = r[..., 0] * r[..., 0] + r[..., 1] * r[..., 1] + r[..., 2] * r[..., 2]
        inv3 = 1.0 / (r2 + e2) ** 1.5
        rf = np.einsum("mnk,nk->mn", r, f)
        out[s:s + block] = c * (np.einsum("mn,nk->mk", (r2 + 2 * e2) * inv3, f)
                                + np.einsum("mn,mnk->mk", rf * inv3, r))
    return out
