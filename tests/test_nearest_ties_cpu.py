"""Tie weights of the nearest-neighbour matrix (Tools/Nearest/nearestMatrix.m).

The reference's stated intent is an interpolation matrix whose tied entries
share 1/k (rows sum to one).  As written, nearestMatrix.m:35-37 pairs the tied
(fine, coarse) entries found in column-major order (find) with the weights
read in row-major order (logical indexing of the transpose), per block of
floor(blockSize 2^27 / (9 Q)) fine points.  Where rows with different tie
counts share a block, weights move to other rows.

oracle/nearest.py restates both: nearest_matrix (1/k, the product default)
and nearest_matrix_reference_order (the code as written).  These tests pin
the second against a hand-worked case, show where the two differ on a tied
lattice and on a prolate spheroid of the batched configuration, and check the
library's ties="reference" option against it bit for bit (host builder, no
GPU needed)."""
import numpy as np
import pytest
import scipy.sparse as sp

import nnkifmm as nk
from oracle.geometry import prolate_spheroid
from oracle.nearest import nearest_matrix, nearest_matrix_reference_order


def test_hand_worked_block():
    """Three fine points, four coarse points, one block: q0 ties with n0 and
    n1 (k = 2), q1 is nearest n2 alone, q2 ties with n1 and n3 (k = 2).
    Column-major pairs: (q0,n0) (q0,n1) (q2,n1) (q1,n2) (q2,n3); row-major
    weights: 1/2 1/2 1 1/2 1/2.  So (q2,n1) gets 1 and (q1,n2) gets 1/2."""
    c = np.array([[-1.0, 0, 0], [1.0, 0, 0], [10.0, 0, 0], [3.0, 0, 0]])
    f = np.array([[0.0, 0, 0], [10.5, 0, 0], [2.0, 0, 0]])
    R = nearest_matrix_reference_order(c, f).toarray()
    expect = np.array([[0.5, 0.5, 0, 0], [0, 0, 0.5, 0], [0, 1.0, 0, 0.5]])
    assert np.array_equal(R, expect)
    S = nearest_matrix(c, f).toarray()
    assert np.array_equal(S.sum(axis=1), [1, 1, 1]) and not np.array_equal(R, S)
    L = nk.nearestMatrix(c, f, blockSize=1.0, builder="host", ties="reference").toarray()
    assert np.array_equal(L, expect)


def tied_lattice():
    g = np.array([[i, j, k] for i in range(5) for j in range(5) for k in range(5)], float) * 0.1
    f = np.concatenate([g[:-1] + 0.05, g + [0.05, 0, 0], g + [0.02, 0.01, 0.0]])
    return g, f


@pytest.mark.parametrize("case", ["lattice", "prolate"])
def test_reference_pairing_differs_from_sharing_only_where_ties_mix(case):
    if case == "lattice":
        c, f = tied_lattice()
    else:
        # a prolate spheroid of the batched configuration (a = 0.6, c = 2):
        # force points at h = 0.1, quadrature at h/4
        c, f = prolate_spheroid(0.6, 2.0, 0.1), prolate_spheroid(0.6, 2.0, 0.025)
    S = nearest_matrix(c, f)
    R = nearest_matrix_reference_order(c, f, block_size=1.0)
    k = S.getnnz(axis=1)
    assert np.array_equal(S.indptr, R.indptr) and np.array_equal(S.indices, R.indices)  # same pattern
    tied = k > 1
    assert tied.any()
    diff = np.abs(S - R).max(axis=1).toarray().ravel()
    rowsum = np.asarray(R.sum(axis=1)).ravel()
    print(case, "coarse", len(c), "fine", len(f), "tied rows", int(tied.sum()), "rows changed",
          int((diff > 0).sum()), "max entry change", diff.max(), "row sums", rowsum.min(), rowsum.max())
    # rows of a block without ties keep weight 1; changes need ties in the block
    assert np.all(rowsum[~tied & (diff == 0)] == 1.0)
    assert (diff > 0).sum() > 0 and (rowsum != 1.0).any()
    # the library's reference pairing, from its own exact tie set, bit for bit
    L = nk.nearestMatrix(c, f, blockSize=1.0, builder="host", ties="reference")
    assert (L != R).nnz == 0 and L.nnz == R.nnz
    # and the default stays the sharing form
    assert (nk.nearestMatrix(c, f, builder="host") != S).nnz == 0


def test_block_size_sets_the_blocks():
    """Small blocks confine the pairing: with one fine point per block the
    reference pairing is the sharing form."""
    c, f = tied_lattice()
    one = 9.0 * len(f) / 2.0 ** 27  # floor(blockSize 2^27 / (9 Q)) = 1
    R1 = nearest_matrix_reference_order(c, f, block_size=one * 1.0000001)
    assert (R1 != nearest_matrix(c, f)).nnz == 0
    L1 = nk.nearestMatrix(c, f, blockSize=one * 1.0000001, builder="host", ties="reference")
    assert (L1 != R1).nnz == 0
    for bs in (0.001, 0.01, 0.3):
        Rb = nearest_matrix_reference_order(c, f, block_size=bs)
        Lb = nk.nearestMatrix(c, f, blockSize=bs, builder="host", ties="reference")
        assert (Lb != Rb).nnz == 0


def test_empty_block_rejected():
    """floor(blockSize 2^27 / (9 Q)) = 0: the reference builds no matrix;
    the library refuses instead of returning an empty one."""
    c, f = tied_lattice()
    tiny = 0.5 * 9.0 * len(f) / 2.0 ** 27
    assert nearest_matrix_reference_order(c, f, block_size=tiny).nnz == 0
    with pytest.raises(nk.NNKError) as e:
        nk.nearestMatrix(c, f, blockSize=tiny, builder="host", ties="reference")
    assert e.value.code == 1 and "blockNodes = 0" in str(e.value)
