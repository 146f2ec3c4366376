"""Adaptive octree with DFS-block node numbering and U/V/W/X interaction
lists, restated from Classes/OcTree.m and Tools/Tree/*.m (FP64).

Test infrastructure only (see oracle/__init__.py).

Node ids are the reference's 1-based ids.  Arrays are indexed by id, with a
dummy row 0, so ``tree.level[i]`` is the level of reference node ``i``.
The list builders follow the reference rules literally (whole-tree scans per
node, O(nodes^2)); they are meant for trees of up to a few thousand nodes.
"""
import sys

import numpy as np
import scipy.sparse as sp

from .mlab import unique_rows_stable, ismember_rows


class MaxDepthError(RuntimeError):
    """OcTree.m:168-170 ``error('Max level reached: Increase Max Depth')``."""


class OcTree:
    def __init__(self, pot_points, target_points, node_capacity=200, max_depth=21,
                 nearest=0, fine_points=None, NN=None, build_lists=True):
        pot_points = np.asarray(pot_points, dtype=np.float64).reshape(-1, 3)
        target_points = np.asarray(target_points, dtype=np.float64).reshape(-1, 3)
        # OcTree.m:80-82
        pts = unique_rows_stable(np.vstack([pot_points, target_points]))
        self.points = pts
        if pot_points is target_points or np.array_equal(pot_points, target_points):
            self.potentials = np.ones(len(pts), dtype=bool) if len(pot_points) else np.zeros(len(pts), bool)
            self.targets = self.potentials.copy()
        else:
            self.potentials = ismember_rows(pts, pot_points)
            self.targets = ismember_rows(pts, target_points)
        n = len(pts)
        self.max_depth = max_depth
        # OcTree.m:97-98: one scalar min and max over all coordinates
        lo = pts.min() if n else 0.0
        hi = pts.max() if n else 0.0
        self._corners = [np.zeros(6), np.array([lo, lo, lo, hi, hi, hi])]
        self._level = [0, 0]
        self._parent = [0, 0]
        self._children = [np.zeros(8, np.int64), np.zeros(8, np.int64)]
        self.node_count = 1
        # OcTree.m:105
        self.node_capacity = min(node_capacity, n - 1)
        self.point_index = np.ones(n, dtype=np.int64)
        self._members = {1: np.arange(n)}
        old = sys.getrecursionlimit()
        sys.setrecursionlimit(max(old, 10000))
        try:
            self._divide([1])
        finally:
            sys.setrecursionlimit(old)
        self.corners = np.array(self._corners)
        self.level = np.array(self._level, dtype=np.int64)
        self.parent = np.array(self._parent, dtype=np.int64)
        self.children = np.array(self._children, dtype=np.int64)
        del self._members
        self.nearest = nearest
        self.fine_points = None if fine_points is None else np.asarray(fine_points, dtype=np.float64)
        # OcTree.m:120-128
        if NN is None and nearest:
            from .nearest import nearest_matrix
            self.NN = nearest_matrix(pot_points, self.fine_points)
        else:
            self.NN = None if NN is None else sp.csr_matrix(NN)
        if build_lists:
            self.gen_interaction_lists()

    # ---------------------------------------------------------------- build
    def _divide(self, nodes):
        """Divide, OcTree.m:155-179: depth check on every visited node, then
        subdivide when the count exceeds the capacity and recurse into the
        new 8-block before moving to the next sibling."""
        for node in nodes:
            if self._level[node] + 1 >= self.max_depth:
                raise MaxDepthError("Max level reached: Increase Max Depth")
            old = self.node_count
            if len(self._members[node]) > self.node_capacity:
                self._divide_node(node)
                self._divide(list(range(old + 1, self.node_count + 1)))

    def _divide_node(self, node):
        """Dividenode, OcTree.m:181-222.  centre = mean([lo;hi]) = (lo+hi)/2;
        child k in 1..8 has bits (x,y,z) = binary(k-1), x most significant;
        a point goes to the upper half iff p > centre (strict)."""
        mem = self._members.pop(node)
        c = self._corners[node]
        lo, hi = c[0:3], c[3:6]
        center = (lo + hi) / 2.0
        p = self.points[mem]
        gt = p > center
        loc = 4 * gt[:, 0] + 2 * gt[:, 1] + gt[:, 2]
        first = self.node_count + 1
        self._children[node] = np.arange(first, first + 8, dtype=np.int64)
        for k in range(8):
            bx, by, bz = (k >> 2) & 1, (k >> 1) & 1, k & 1
            nlo = np.array([center[0] if bx else lo[0], center[1] if by else lo[1], center[2] if bz else lo[2]])
            nhi = np.array([hi[0] if bx else center[0], hi[1] if by else center[1], hi[2] if bz else center[2]])
            self._corners.append(np.concatenate([nlo, nhi]))
            self._level.append(self._level[node] + 1)
            self._parent.append(node)
            self._children.append(np.zeros(8, np.int64))
            sel = mem[loc == k]
            self._members[first + k] = sel
            self.point_index[sel] = first + k
        self.node_count += 8

    # ------------------------------------------------------------ predicates
    def ids(self):
        return np.arange(1, self.node_count + 1)

    def is_leaf_all(self, idx):
        """isleaf(...,'All'), Tools/Tree/isleaf.m:18-20."""
        return self.children[np.asarray(idx), 0] == 0

    def is_leaf_target(self, idx):
        """isleaf(...,'Target'): the id occurs in pointIndex(targets); isleaf.m:14-15."""
        s = np.zeros(self.node_count + 1, dtype=bool)
        s[self.point_index[self.targets]] = True
        return s[np.asarray(idx)]

    def is_leaf_potential(self, idx):
        """isleaf(...,'Potential'); isleaf.m:16-17."""
        s = np.zeros(self.node_count + 1, dtype=bool)
        s[self.point_index[self.potentials]] = True
        return s[np.asarray(idx)]

    def intersects(self, i, idx):
        """Closed-box touch/overlap test, Tools/Tree/nodeintersection.m:14-22."""
        c1 = self.corners[i]
        c2 = self.corners[np.asarray(idx)]
        return ~((c2[..., 0] > c1[3]) | (c2[..., 3] < c1[0]) | (c2[..., 1] > c1[4]) |
                 (c2[..., 4] < c1[1]) | (c2[..., 2] > c1[5]) | (c2[..., 5] < c1[2]))

    def get_children(self, idx):
        """getChildren, Tools/Tree/getChildren.m:10-17, including its quirk:
        when no input is a non-leaf the result is empty (the input leaves are
        dropped too)."""
        idx = np.asarray(idx, dtype=np.int64).ravel()
        if idx.size == 0:
            return idx
        leaf = self.is_leaf_all(idx)
        new = self.children[idx[~leaf]].T.reshape(-1)  # column-major reshape
        if new.size == 0:
            return np.zeros(0, np.int64)
        return np.concatenate([idx[leaf], new, self.get_children(new)])

    # ----------------------------------------------------------------- lists
    def _uvw(self, i):
        """genUVWinterationlists, OcTree.m:307-366."""
        allids = self.ids()
        lvl = self.level[i]
        tleaf = self.is_leaf_target(i)
        pot_leaf_all = self.is_leaf_potential(allids)
        touch_i = self.intersects(i, allids)
        # U, :323-327
        U = allids[touch_i & pot_leaf_all] if tleaf else np.zeros(0, np.int64)
        # V, :330-339
        par = self.parent[i]
        pn = allids[self.intersects(par, allids) & (lvl - 1 >= self.level[1:])]
        pn = np.setdiff1d(pn, np.concatenate([self.parent[pn], [par]]))
        pn = pn[~self.is_leaf_all(pn)]
        pnc = self.children[pn].T.reshape(-1)
        pnc = pnc[~self.intersects(i, pnc)] if pnc.size else pnc
        V = np.setdiff1d(pnc, U)
        # W, :343-365
        if tleaf:
            nb = allids[touch_i & (lvl >= self.level[1:])]
            nb = np.setdiff1d(nb, self.parent[nb])
            nbc = self.get_children(nb)
            nbc = nbc[self.is_leaf_potential(nbc)] if nbc.size else nbc
            W0 = np.setdiff1d(nbc, U)
            inW = np.zeros(self.node_count + 1, dtype=bool)
            inW[W0] = True
            # Merge loop :352-360.  Each merge is W = [setdiff(W,children); node],
            # so W stays sorted except for the most recently merged node, which
            # sits at the end.  Merges within one level touch disjoint children
            # and are applied together; nodes of a level run in ascending id, so
            # the last merge of a level is its largest merged id.
            last = 0
            maxl = int(self.level[1:].max())
            for level in range(maxl, 0, -1):
                nodes = allids[(self.level[1:] == level) & (self.children[1:, 0] != 0)]
                if nodes.size == 0:
                    continue
                ok = inW[self.children[nodes]].all(axis=1)
                merged = nodes[ok]
                if merged.size:
                    inW[self.children[merged]] = False
                    inW[merged] = True
                    last = int(merged.max())
            W = np.nonzero(inW)[0].astype(np.int64)
            if last:
                W = np.concatenate([W[W != last], [last]])
        else:
            W = np.zeros(0, np.int64)
        return U.astype(np.int64), V.astype(np.int64), W

    def gen_interaction_lists(self):
        """geninteractionlists, OcTree.m:265-290.  X(i) is the row list of
        ``find(Wpadded == i)``: column-major, i.e. ordered by the position of
        i inside W(j) first and by j second."""
        nc = self.node_count
        self.U = [np.zeros(0, np.int64) for _ in range(nc + 1)]
        self.V = [np.zeros(0, np.int64) for _ in range(nc + 1)]
        self.W = [np.zeros(0, np.int64) for _ in range(nc + 1)]
        self.X = [np.zeros(0, np.int64) for _ in range(nc + 1)]
        for i in range(2, nc + 1):
            self.U[i], self.V[i], self.W[i] = self._uvw(i)
        entries = []
        for j in range(1, nc + 1):
            for pos, i in enumerate(self.W[j]):
                entries.append((int(i), pos, j))
        entries.sort()
        for i, pos, j in entries:
            self.X[i] = np.append(self.X[i], j)

    # --------------------------------------------------------------- export
    def leaf_of_points(self):
        return self.point_index.copy()
