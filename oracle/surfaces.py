"""KIFMM equivalent / check surfaces (FP64).

Test infrastructure only (see oracle/__init__.py).
"""
import numpy as np

from .mlab import linspace, meshgrid3_colmajor


def _shell(lo, hi, res, shells):
    x = linspace(lo[0], hi[0], res)
    y = linspace(lo[1], hi[1], res)
    z = linspace(lo[2], hi[2], res)
    X, Y, Z, j, i, k = meshgrid3_colmajor(x, y, z)
    inner = lambda a: (a >= shells) & (a <= res - 1 - shells)
    interior = inner(j) & inner(i) & inner(k)
    return np.stack([X[~interior], Y[~interior], Z[~interior]], axis=1)


def upsurf(corners, res=6, shells=1):
    """Points of the node box's outer lattice shells; Tools/KIFMM/genupsurf.m:20-37.
    ``corners`` = [x1 y1 z1 x2 y2 z2] (OcTree.m:36-39)."""
    c = np.asarray(corners, dtype=np.float64)
    return _shell(c[0:3], c[3:6], res, shells)


def downsurf(corners, res=6, shells=1):
    """Same lattice on the 3x box [lo-w, hi+w]; Tools/KIFMM/gendownsurf.m:21-39."""
    c = np.asarray(corners, dtype=np.float64)
    w = c[3:6] - c[0:3]
    return _shell(c[0:3] - w, c[3:6] + w, res, shells)


def surface_count(res=6, shells=1):
    inner = max(res - 2 * shells, 0)
    return res ** 3 - inner ** 3
