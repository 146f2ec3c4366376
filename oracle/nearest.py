"""Nearest-neighbour force-to-quadrature matrix (FP64).

Test infrastructure only (see oracle/__init__.py).
"""
import numpy as np
import scipy.sparse as sp


def nearest_matrix(coarse, fine, block=2048):
    """NN (Q x N) of Tools/Nearest/nearestMatrix.m:17-41.

    For each fine point q, d2(q,n) = (dx^2 + dy^2) + dz^2 in FP64
    (``sum((fine-coarse).^2,3)``, :30-33; products and sums rounded one at a
    time, no fused multiply-add), and NN(q,n) = [d2 == min_n d2] / #ties
    (:34-37), so a fine point equidistant from k coarse points gives 1/k to
    each.  Rows sum to one.
    """
    coarse = np.asarray(coarse, dtype=np.float64).reshape(-1, 3)
    fine = np.asarray(fine, dtype=np.float64).reshape(-1, 3)
    Q, N = fine.shape[0], coarse.shape[0]
    rows, cols, vals = [], [], []
    for s in range(0, Q, block):
        f = fine[s:s + block]
        dx = f[:, 0:1] - coarse[:, 0][None, :]
        dy = f[:, 1:2] - coarse[:, 1][None, :]
        dz = f[:, 2:3] - coarse[:, 2][None, :]
        d2 = (dx * dx + dy * dy) + dz * dz
        mn = d2.min(axis=1, keepdims=True)
        eq = d2 == mn
        cnt = eq.sum(axis=1)
        r, c = np.nonzero(eq)
        rows.append(r + s)
        cols.append(c)
        vals.append(1.0 / cnt[r])
    if Q == 0:
        return sp.csr_matrix((0, N))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(Q, N))
