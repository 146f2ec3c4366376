"""MATLAB built-in semantics that the reference relies on, restated in numpy.

Test infrastructure only (see oracle/__init__.py).
"""
import numpy as np


def linspace(d1, d2, n):
    """MATLAB ``linspace(d1,d2,n)`` for finite arguments:
    ``y = d1 + (0:n-1).*(d2-d1)./(n-1)`` with both end points set exactly.

    numpy's linspace rounds differently (``start + k*(delta/div)``); the
    reference surfaces (Tools/KIFMM/genupsurf.m:38-40) and the sphere generator
    (Geometries/Sphere.m:17) use the MATLAB form.
    """
    n = int(np.floor(n))
    if n <= 0:
        return np.zeros(0)
    if n == 1:
        return np.array([float(d2)])
    n1 = n - 1
    k = np.arange(n, dtype=np.float64)
    y = d1 + (k * (d2 - d1)) / n1
    if d1 == d2:
        y[:] = d1
    else:
        y[0] = d1
        y[-1] = d2
    return y


def meshgrid3_colmajor(x, y, z):
    """``[X,Y,Z] = meshgrid(x,y,z)`` followed by column-major ``(:)``:
    the y index runs fastest, then x, then z.  Returns three flat arrays and
    the (j, i, k) index triplets (y, x, z indices) of each entry."""
    ny, nx, nz = len(y), len(x), len(z)
    k, i, j = np.meshgrid(np.arange(nz), np.arange(nx), np.arange(ny), indexing="ij")
    j = j.ravel(); i = i.ravel(); k = k.ravel()
    return x[i], y[j], z[k], j, i, k


def unique_rows_stable(a):
    """``unique(a,'rows','stable')``: first occurrences, original order.
    Rows compare by value (so -0.0 equals 0.0, as in MATLAB)."""
    seen = {}
    keep = []
    for r in range(a.shape[0]):
        key = tuple(float(v) + 0.0 for v in a[r])
        if key not in seen:
            seen[key] = r
            keep.append(r)
    return a[np.array(keep, dtype=np.int64)] if keep else a[:0]


def ismember_rows(a, b):
    """``ismember(a,b,'rows')`` as a boolean mask over the rows of a."""
    s = {tuple(float(v) + 0.0 for v in row) for row in b}
    return np.array([tuple(float(v) + 0.0 for v in row) in s for row in a], dtype=bool)
