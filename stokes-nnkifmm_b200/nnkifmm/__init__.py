"""B200 KIFMM for regularized Stokeslets with nearest-neighbour quadrature,
and the GMRES mobility solve that calls it.

Host mirror of the Stokes-NNKIFMM MATLAB API (Classes/OcTree.m,
Classes/KIFMM.m, Classes/Swimmers.m, Mobility/*.m) over the C ABI of
libnnkifmm.so (include/nnkifmm.h).  All FMM work runs on the GPU; the
library refuses to create an FMM without a CUDA device.
"""
from ._lib import (NNKError, MaxDepthError, NoConvergence, context, lib, LIB_PATH,  # noqa: F401
                   LAYOUT_ROWS, LAYOUT_BLOCKED, PREC_FP64, PREC_MIXED, PREC_NEAR32)
from .octree import OcTree, nearestMatrix  # noqa: F401
from .kifmm import KIFMM  # noqa: F401
from .mobility import (Swimmers, Mobility, hegedus, mobilityProblem, mobilityProblemGravity,  # noqa: F401
                       mobilityRHS, richardson)
from .batch import BatchMobility  # noqa: F401
from .resistance import Gen_Resistance, Rigid_Resistance, velocityModes  # noqa: F401
