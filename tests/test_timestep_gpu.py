"""The caller of the solve: time stepping of the swimmers' positions and
orientations (Data Generation/Squiremers.m:47-54 integrates
mobilityProblem with ode45; here scipy's RK45 calls mobilityProblem, which
rebuilds the tree and the FMM at every evaluation as the reference does).
A free squirmer with slip B1 sin(t) e_t swims along its axis at 2 B1 / 3
(Blake's squirmer speed for a unit sphere) without rotating."""
import numpy as np
import pytest
from scipy.integrate import solve_ivp

import nnkifmm as nk
from nnkifmm.workloads import cube_sphere, squirmer_slip

pytestmark = pytest.mark.gpu


def test_free_squirmer_speed_and_integration():
    body, fine = cube_sphere(1.0, (0, 0, 0), 10), cube_sphere(1.0, (0, 0, 0), 40)
    NN = nk.nearestMatrix(body, fine)
    sw = nk.Swimmers()
    sw.addSwimmer(body, fine, NN, [0, 0, 0], [1, 0, 0, 0, 1, 0], squirmer_slip(body, 1.0, 0.0), [0, 0, 0],
                  [0, 0, 0])
    calls = []

    def rhs(t, x):
        calls.append(t)
        return nk.mobilityProblem(sw, None, t, x, [0.01, 1.0], {"nodeCapacity": 60, "nearest": 1}, tol=1e-8,
                                  maxIter=300)

    x0 = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], float)
    v = rhs(0.0, x0)
    # swims along b3 = e_z at 2/3 (discretization error ~1%), no drift, no rotation
    assert abs(v[2] / (2.0 / 3.0) - 1) < 3e-2, v[2]
    assert np.abs(v[[0, 1]]).max() < 1e-3 * abs(v[2]) and np.abs(v[3:]).max() < 1e-3 * abs(v[2])
    T = 0.3
    sol = solve_ivp(rhs, (0.0, T), x0, method="RK45", rtol=1e-6, atol=1e-9)
    assert sol.success and len(calls) > 6
    xT = sol.y[:, -1]
    # a rigid translation: the centre moves by v T, the basis stays put
    assert abs(xT[2] - v[2] * T) < 1e-4 and np.allclose(xT[3:], x0[3:], atol=1e-4)
