"""GMRES with the semantics MATLAB's gmres is called with in the reference
(Mobility/mobilityProblem.m:53,57; Data Generation/DirectMethodComparison.m:28):
x0 = 0, restart = [] (unrestarted), stop at ||b - A x|| / ||b|| <= tol.

MATLAB's gmres itself is closed source and not part of the reference; its
iterates are not pinned.  This restatement uses Householder-free modified
Gram-Schmidt with one reorthogonalisation pass and Givens rotations.

Test infrastructure only (see oracle/__init__.py).
"""
import numpy as np


def gmres(afun, b, restart=None, tol=1e-6, maxit=None, post=None):
    b = np.asarray(b, dtype=np.float64).ravel()
    n = b.size
    if maxit is None:
        maxit = min(n, 10)
    m = restart if restart else maxit
    m = min(m, n)
    x = np.zeros(n)
    nb = np.linalg.norm(b)
    if nb == 0:
        return (post(x) if post else x), 0, 0.0, 0, [0.0]
    r = b.copy()
    beta = nb
    total = 0
    resvec = [nb]
    while True:
        V = np.zeros((m + 1, n))
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        V[0] = r / beta
        k = 0
        for j in range(m):
            if total >= maxit:
                break
            w = afun(V[j])
            for _ in range(2):
                h = V[:j + 1] @ w
                w = w - V[:j + 1].T @ h
                H[:j + 1, j] += h
            H[j + 1, j] = np.linalg.norm(w)
            if H[j + 1, j] > 0:
                V[j + 1] = w / H[j + 1, j]
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            den = np.hypot(H[j, j], H[j + 1, j])
            cs[j] = H[j, j] / den if den > 0 else 1.0
            sn[j] = H[j + 1, j] / den if den > 0 else 0.0
            H[j, j] = den
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            total += 1
            k = j + 1
            resvec.append(abs(g[j + 1]))
            if abs(g[j + 1]) / nb <= tol:
                break
        if k:
            y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
            x = x + V[:k].T @ y
        r = b - afun(x)
        beta = np.linalg.norm(r)
        if beta / nb <= tol or total >= maxit or k == 0:
            break
    relres = beta / nb
    flag = 0 if relres <= tol else 1
    if post:
        x = post(x)
    return x, flag, relres, total, resvec
