"""CPU FP64 restatement of the Stokes-NNKIFMM reference (MATLAB) for the KIFMM
matvec and the GMRES mobility solve.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library and its
Python binding under ``stokes-nnkifmm_b200/``) imports, links or executes this
package.  Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline``
/ ``--impl reference`` legs of ``bench.py`` use it, and only as the reference
answer the GPU results are compared with, or as the timed CPU baseline.

Parity status.  The reference is 100 % MATLAB and cannot run on this machine
(no MATLAB, no Octave), and it ships no golden vectors.  The only known answer
it holds is the Stokes drag of a unit sphere, ``F = 6*pi*mu*a*U``
(Data Generation/DirectMethodComparison.m:34), which ``tests/test_oracle_*``
check against this restatement within discretisation error.  Exact-value
parity against the reference is therefore *unpinned*: the restatement follows
the cited MATLAB lines operation by operation (FP64, same op order where it
matters for ties and tree splits), and the GPU path is checked against it.

Modules
  kernel    -- regularized Stokeslet matrix and block products (Tools/kernel.m,
               Tools/Other/blockcomputation.m, Tools/Nearest/nearestBlockComputation.m)
  mlab      -- MATLAB built-in semantics used by the reference (linspace,
               unique(...,'rows','stable'), ismember rows, meshgrid order)
  geometry  -- point generators (Geometries/*.m)
  surfaces  -- KIFMM equivalent/check surfaces (Tools/KIFMM/*.m)
  nearest   -- nearest-neighbour matrix (Tools/Nearest/nearestMatrix.m)
  octree    -- adaptive octree and U/V/W/X lists (Classes/OcTree.m, Tools/Tree/*.m)
  kifmm     -- upward/downward passes, reduced pass/solve (Tools/Passes/*.m,
               Tools/Nearest/*Nearest.m, Mobility/ReducedSolve.m, Classes/KIFMM.m)
  gmres     -- unrestarted GMRES with relative-residual stop (MATLAB gmres semantics)
  mobility  -- Swimmers assembly, B/BT/A1/A2, mobility matvec, preconditioner,
               mobilityProblem, the dense FP64 system (Classes/Swimmers.m, Mobility/*.m)
  gradient  -- dense FP64 adjoint gradient of a rigid-velocity loss
  parfor    -- the kifmm matvec with the reference's parfor loops over the nodes
               of a level on worker processes (upwardPass.m:40, downwardPass.m:45,177)
"""
