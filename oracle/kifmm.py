"""KIFMM matvec in the reference's own structure (FP64): per-level loops over
nodes, with the surface kernel matrix built and solved by LU for every node
on every pass, as Tools/Passes/{upwardPass,downwardPass,Up,DownNonleaf,
Downleaf}.m and their Tools/Nearest/*Nearest.m variants do.

Test infrastructure only (see oracle/__init__.py).
"""
import numpy as np
import scipy.linalg as sla

from .kernel import kernel, apply_kernel
from .surfaces import upsurf, downsurf, surface_count


class KIFMM:
    """Classes/KIFMM.m:46-61.  ``fmt`` 1 = interleaved [x1 y1 z1 x2 ...]',
    2 = blocked [x1..xN y1..yN z1..zN]' (used when ``gmres`` is 1)."""

    def __init__(self, tree, eps, mu, corona_res=6, corona_shells=1, gmres=0, fmt=1):
        self.tree = tree
        self.eps = float(eps)
        self.mu = float(mu)
        self.res = corona_res
        self.shells = corona_shells
        self.gmres = gmres
        self.fmt = fmt

    # KIFMM.m:83-89 / :97-103
    def _to_rows(self, v):
        if self.gmres == 1:
            v = np.asarray(v, dtype=np.float64).ravel()
            return v.reshape(-1, 3) if self.fmt == 1 else v.reshape(3, -1).T
        return np.asarray(v, dtype=np.float64).reshape(-1, 3)

    def _from_rows(self, v):
        if self.gmres == 1:
            return v.reshape(-1) if self.fmt == 1 else v.T.reshape(-1)
        return v

    def compute_vel(self, potentials):
        """KIFMM.computeVel, KIFMM.m:63-105."""
        pot = self._to_rows(potentials)
        up = upward_pass(self.tree, pot, self.eps, self.mu, self.res, self.shells)
        vel = downward_pass(self.tree, pot, up, self.eps, self.mu, self.res, self.shells)
        return self._from_rows(vel)

    def compute_vel_sparse(self, potentials):
        """KIFMM.computeVelSparse, KIFMM.m:107-155: coronaRes 4 (56 points).
        The reference's restore of coronaShells has a typo (``corornaShells``,
        :138,145) with no effect on the result; shells stay as configured."""
        pot = self._to_rows(potentials)
        up = upward_pass(self.tree, pot, self.eps, self.mu, 4, self.shells)
        vel = downward_pass(self.tree, pot, up, self.eps, self.mu, 4, self.shells)
        return self._from_rows(vel)

    def reduced_compute_vel(self, potentials):
        """KIFMM.reducedComputeVel, KIFMM.m:157-198 (Tools/Passes/reducedPass.m)."""
        pot = self._to_rows(potentials)
        return self._from_rows(reduced_pass(self.tree, pot, self.eps, self.mu))

    def reduced_solve(self, vel):
        """KIFMM.reducedSolve, KIFMM.m:200-242 (Mobility/ReducedSolve.m)."""
        v = self._to_rows(vel)
        return self._from_rows(reduced_solve(self.tree, v, self.eps, self.mu))


def _leaf_sources(tree, node, pot):
    """Sources of leaf ``node`` and their force densities.

    Plain mode: the potential points of the leaf (upwardPass.m:54-77).
    NEAREST mode: the fine points with a nonzero NN entry in the leaf's
    columns, ascending, carrying kron(NN_sub, I3)*f (upwardPass.m:58-66,
    nearestBlockComputation.m:26-29).  As in downwardPass.m:92,221 the
    NEAREST gather slices columns by ``pointIndex == node`` over all points,
    which presumes potentials and targets are the same set.
    """
    if tree.nearest:
        cols = np.nonzero(tree.point_index == node)[0]
        sub = tree.NN[:, cols]
        rows = np.nonzero(np.asarray(abs(sub).sum(axis=1)).ravel() != 0)[0]
        NNs = sub[rows]
        g = NNs @ pot[cols]
        return tree.fine_points[rows], np.asarray(g)
    pmask = tree.point_index[tree.potentials] == node
    return tree.points[tree.potentials][pmask], pot[pmask]


def up_node(tree, node, pot, uppot, eps, mu, res, shells, pot_leaf):
    """One iteration of upwardPass.m's parfor over the nodes of a level
    (:40-98; Up.m:31-33): the check potential on the node's downsurf from its
    leaf sources or its children's equivalent densities, then
    kernel(upsurf, downsurf) \\ check."""
    us = upsurf(tree.corners[node], res, shells)
    ds = downsurf(tree.corners[node], res, shells)
    if pot_leaf:
        src, g = _leaf_sources(tree, node, pot)
        check = apply_kernel(src, ds, g, eps, mu)
    else:
        ch = tree.children[node]
        csurf = np.concatenate([upsurf(tree.corners[c], res, shells) for c in ch])
        cpot = np.concatenate([uppot[c].reshape(-1, 3) for c in ch])
        check = apply_kernel(csurf, ds, cpot, eps, mu)
    K = kernel(us, ds, eps, mu)
    return sla.solve(K, check.reshape(-1))


def up_levels(tree, res, shells):
    """Per level, from the deepest to the root, the nodes upwardPass.m visits:
    the non-empty potential leaves and the non-leaves (:33-35), with their
    leaf flags."""
    ids = tree.ids()
    pot_leaf = tree.is_leaf_potential(ids)
    nonleaf = ~tree.is_leaf_all(ids)
    out = []
    for level in range(int(tree.level[1:].max()), -1, -1):
        sel = (tree.level[1:] == level) & (pot_leaf | nonleaf)
        out.append((ids[sel], pot_leaf[sel]))
    return out


def upward_pass(tree, pot, eps, mu, res=6, shells=1):
    """Tools/Passes/upwardPass.m:18-99.  Levels max..0; nodes of a level are
    the non-empty potential leaves and the non-leaves (:33-35); returns
    uppot[(nodeCount+1), 3P] with rows [x y z] interleaved per surface point."""
    P = surface_count(res, shells)
    uppot = np.zeros((tree.node_count + 1, 3 * P))
    for nodes, leaf in up_levels(tree, res, shells):
        for node, pl in zip(nodes, leaf):
            uppot[node] = up_node(tree, node, pot, uppot, eps, mu, res, shells, pl)
    return uppot


def down_node(tree, node, pot, uppot, downpot, eps, mu, res, shells):
    """One iteration of downwardPass.m's parfor over the nodes of a level
    (:45-166; DownNonleaf.m:42-46): the check potential on the node's upsurf
    from V (M2L), X (P2L) and the parent's downsurf (L2L), then
    kernel(downsurf, upsurf) \\ check."""
    P = surface_count(res, shells)
    us = upsurf(tree.corners[node], res, shells)
    ds = downsurf(tree.corners[node], res, shells)
    rhs = np.zeros((P, 3))
    v = tree.V[node]
    if len(v):
        vs = np.concatenate([upsurf(tree.corners[k], res, shells) for k in v])
        vp = np.concatenate([uppot[k].reshape(-1, 3) for k in v])
        rhs += apply_kernel(vs, us, vp, eps, mu)
    for xn in tree.X[node]:
        src, g = _leaf_sources(tree, xn, pot)
        if len(src):
            rhs += apply_kernel(src, us, g, eps, mu)
    par = tree.parent[node]
    ps = downsurf(tree.corners[par], res, shells)
    rhs += apply_kernel(ps, us, downpot[par].reshape(-1, 3), eps, mu)
    K = kernel(ds, us, eps, mu)
    return sla.solve(K, rhs.reshape(-1))


def leaf_velocity(tree, node, pot, uppot, downpot, eps, mu, res, shells):
    """One iteration of downwardPass.m's parfor over the target leaves
    (:177-294): L2T + U (P2P) + W (M2T); returns the leaf's target mask and
    velocities."""
    targets = tree.points[tree.targets]
    tmask = tree.point_index[tree.targets] == node
    tp = targets[tmask]
    ds = downsurf(tree.corners[node], res, shells)
    u = apply_kernel(ds, tp, downpot[node].reshape(-1, 3), eps, mu)
    for un in tree.U[node]:
        src, g = _leaf_sources(tree, un, pot)
        if len(src):
            u += apply_kernel(src, tp, g, eps, mu)
    w = tree.W[node]
    if len(w):
        ws = np.concatenate([upsurf(tree.corners[k], res, shells) for k in w])
        wp = np.concatenate([uppot[k].reshape(-1, 3) for k in w])
        u += apply_kernel(ws, tp, wp, eps, mu)
    return tmask, u


def down_levels(tree):
    """The nodes of levels 1..max (downwardPass.m:39-44; the root's downward
    expansion is zero) and the non-empty target leaves (:170-176)."""
    ids = tree.ids()
    levels = [ids[tree.level[1:] == level] for level in range(1, int(tree.level[1:].max()) + 1)]
    return levels, ids[tree.is_leaf_target(ids)]


def downward_pass(tree, pot, uppot, eps, mu, res=6, shells=1):
    """Tools/Passes/downwardPass.m:23-306.  Levels 1..max over all nodes
    (root downpot = 0): check potential on the node's upsurf from V (M2L),
    X (P2L) and the parent's downsurf (L2L), then kernel(downsurf,upsurf)\\RHS.
    Then for every non-empty target leaf: L2T + U (P2P) + W (M2T)."""
    P = surface_count(res, shells)
    downpot = np.zeros((tree.node_count + 1, 3 * P))
    levels, leaves = down_levels(tree)
    for nodes in levels:
        for node in nodes:
            downpot[node] = down_node(tree, node, pot, uppot, downpot, eps, mu, res, shells)
    vel = np.zeros((int(tree.targets.sum()), 3))
    for node in leaves:
        tmask, u = leaf_velocity(tree, node, pot, uppot, downpot, eps, mu, res, shells)
        vel[tmask] = u
    return vel


def _leaf_block(tree, node, eps, mu):
    """Leaf self-interaction matrix: S(fine->targets)*kron(NN_sub,I3) in
    NEAREST mode (ReducedSolve.m:96-111), S(points->targets) otherwise."""
    targets = tree.points[tree.targets]
    tmask = tree.point_index[tree.targets] == node
    tp = targets[tmask]
    if tree.nearest:
        sub = tree.NN[:, tmask]
        rows = np.nonzero(np.asarray(abs(sub).sum(axis=1)).ravel() != 0)[0]
        NNs = sub[rows].toarray()
        S = kernel(tree.fine_points[rows], tp, eps, mu)
        return S @ np.kron(NNs, np.eye(3)), tmask
    src = tree.points[tree.potentials][tree.point_index[tree.potentials] == node]
    return kernel(src, tp, eps, mu), tmask


def reduced_pass(tree, pot, eps, mu):
    """Leaf-local self interaction only; Tools/Passes/reducedPass.m:21-81."""
    ids = tree.ids()
    vel = np.zeros((int(tree.targets.sum()), 3))
    for node in ids[tree.is_leaf_target(ids)]:
        A, tmask = _leaf_block(tree, node, eps, mu)
        vel[tmask] = (A @ pot[tmask].reshape(-1)).reshape(-1, 3)
    return vel


def reduced_solve(tree, vel, eps, mu):
    """Per-leaf direct solve (S_leaf*NN_leaf) \\ u_leaf; Mobility/ReducedSolve.m:86-134."""
    ids = tree.ids()
    out = np.zeros((int(tree.targets.sum()), 3))
    for node in ids[tree.is_leaf_target(ids)]:
        A, tmask = _leaf_block(tree, node, eps, mu)
        out[tmask] = sla.solve(A, vel[tmask].reshape(-1)).reshape(-1, 3)
    return out
