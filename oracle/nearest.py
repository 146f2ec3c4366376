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


def nearest_matrix_reference_order(coarse, fine, block_size=1.0):
    """NN exactly as Tools/Nearest/nearestMatrix.m:17-41 is written, tie
    weights included.

    The fine points are cut into blocks of
    blockNodes = floor(blockSize * 2^27 / (9 Q)) rows (:23-24); none when
    that is 0, and NN is then empty.  Per block (:30-39):
      [Ir, Ic] = find(d2 == A)          -> the tied (q, n) pairs in
                                           column-major order (by n, then q);
      values((d2 == A)')                -> their weights 1/k_q read through
                                           the transpose, i.e. in row-major
                                           order (by q, then n);
    and the j-th pair receives the j-th weight.  Without ties both orders
    coincide (every weight is 1).  In a block where rows with different
    tie counts k_q meet, weights land on other rows: rows no longer sum to
    one.  sparse(rows, cols, weight, Q, N) keeps the pairs (:41).
    """
    coarse = np.asarray(coarse, dtype=np.float64).reshape(-1, 3)
    fine = np.asarray(fine, dtype=np.float64).reshape(-1, 3)
    Q, N = fine.shape[0], coarse.shape[0]
    if Q == 0:
        return sp.csr_matrix((0, N))
    block_nodes = int(np.floor(block_size * 2.0 ** 27 / (9.0 * Q)))
    rows, cols, vals = [], [], []
    for s in range(0, Q if block_nodes > 0 else 0, max(block_nodes, 1)):
        f = fine[s:s + block_nodes]
        dx = f[:, 0:1] - coarse[:, 0][None, :]
        dy = f[:, 1:2] - coarse[:, 1][None, :]
        dz = f[:, 2:3] - coarse[:, 2][None, :]
        d2 = (dx * dx + dy * dy) + dz * dz
        eq = d2 == d2.min(axis=1, keepdims=True)
        ic, ir = np.nonzero(eq.T)                      # find(d2 == A): column-major
        values = (eq / eq.sum(axis=1, keepdims=True))  # (d2 == A) ./ sum(d2 == A, 2)
        weight = values[eq]                            # values((d2 == A)'): row-major
        rows.append(ir + s)
        cols.append(ic)
        vals.append(weight)
    if not rows:
        return sp.csr_matrix((Q, N))
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(Q, N))
