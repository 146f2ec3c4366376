"""The oracle's KIFMM matvec with the reference's parfor loops: the nodes of a
level in the upward pass (upwardPass.m:40), in the downward pass
(downwardPass.m:45) and the target leaves (downwardPass.m:177) run on a pool
of worker processes, as MATLAB runs them on `parThreads` workers
(KIFMM.m:15,52); each worker does its LU and BLAS calls on one thread, like a
MATLAB pool worker.  The per-node work is the serial oracle's own
(oracle/kifmm.py: up_node, down_node, leaf_velocity), so results agree with it
to rounding.  The expansions live in shared memory; levels are barriers.

Test infrastructure only (see oracle/__init__.py): the reference arm of the
benchmark times it.  The pool is started with `spawn`.
"""
import multiprocessing as mp
import os
from multiprocessing import shared_memory

import numpy as np

from .kifmm import down_levels, down_node, leaf_velocity, up_levels, up_node
from .surfaces import surface_count

_W = {}  # worker state: tree, parameters and the shared arrays


def _shared(shape):
    shm = shared_memory.SharedMemory(create=True, size=max(int(np.prod(shape)) * 8, 8))
    return shm, np.ndarray(shape, np.float64, buffer=shm.buf)


def _init(tree, params, layout):
    _W["tree"] = tree
    _W["p"] = params
    for key, (name, shape) in layout.items():
        shm = shared_memory.SharedMemory(name=name)  # spawned workers share the parent's resource tracker
        _W[key + "_shm"] = shm
        _W[key] = np.ndarray(shape, np.float64, buffer=shm.buf)


def _up(job):
    nodes, leaf = job
    eps, mu, res, shells = _W["p"]
    for node, pl in zip(nodes, leaf):
        _W["uppot"][node] = up_node(_W["tree"], node, _W["pot"], _W["uppot"], eps, mu, res, shells, pl)


def _down(nodes):
    eps, mu, res, shells = _W["p"]
    for node in nodes:
        _W["downpot"][node] = down_node(_W["tree"], node, _W["pot"], _W["uppot"], _W["downpot"],
                                        eps, mu, res, shells)


def _leaves(nodes):
    eps, mu, res, shells = _W["p"]
    for node in nodes:
        tmask, u = leaf_velocity(_W["tree"], node, _W["pot"], _W["uppot"], _W["downpot"], eps, mu, res, shells)
        _W["vel"][tmask] = u


def _chunks(a, n):
    """Contiguous slices of a, at most n of them, none empty."""
    k = max(1, min(n, len(a)))
    return [c for c in np.array_split(np.asarray(a), k) if len(c)]


class ParforKIFMM:
    """KIFMM.computeVel (KIFMM.m:63-105) with `workers` pool workers; forces
    and velocities as (n, 3) rows.  close() ends the pool."""

    def __init__(self, tree, eps, mu, workers, res=6, shells=1):
        self.tree, self.workers = tree, int(workers)
        P = surface_count(res, shells)
        nc = tree.node_count
        npot, ntgt = int(tree.potentials.sum()), int(tree.targets.sum())
        shapes = {"pot": (npot, 3), "uppot": (nc + 1, 3 * P), "downpot": (nc + 1, 3 * P), "vel": (ntgt, 3)}
        self._shm, self._arr = {}, {}
        for key, shape in shapes.items():
            self._shm[key], self._arr[key] = _shared(shape)
        layout = {k: (self._shm[k].name, shapes[k]) for k in shapes}
        # one BLAS/OpenMP thread per worker: the spawned interpreters read these
        # when they load numpy
        saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
        try:
            for k in saved:
                os.environ[k] = "1"
            self.pool = mp.get_context("spawn").Pool(self.workers, initializer=_init,
                                                     initargs=(tree, (float(eps), float(mu), res, shells), layout))
        finally:
            for k, v in saved.items():
                if v is None:
                    os.environ.pop(k, None)
                else:
                    os.environ[k] = v
        self._levels_up = up_levels(tree, res, shells)
        self._levels_down, self._leaves = down_levels(tree)

    def compute_vel(self, pot):
        a = self._arr
        a["pot"][:] = np.asarray(pot, np.float64).reshape(-1, 3)
        a["uppot"][:] = 0.0
        a["downpot"][:] = 0.0
        a["vel"][:] = 0.0
        n = 4 * self.workers  # a few slices per worker per level, for balance
        for nodes, leaf in self._levels_up:
            jobs = [(nodes[s], leaf[s]) for s in _chunks(np.arange(len(nodes)), n)]
            self.pool.map(_up, jobs)
        for nodes in self._levels_down:
            self.pool.map(_down, _chunks(nodes, n))
        self.pool.map(_leaves, _chunks(self._leaves, n))
        return a["vel"].copy()

    def close(self):
        self.pool.close()
        self.pool.join()
        self._arr = {}  # the views go before their blocks
        for shm in self._shm.values():
            shm.close()
            shm.unlink()
        self._shm = {}
