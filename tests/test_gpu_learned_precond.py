"""GPU: the learned Davidson preconditioner (dft_eig_opts.preconditioner = -3).

The reference corrects with the diagonal of H - theta (davidsonCorrection,
EigenvalueSolverMolecule.cpp:521-555).  Here the correction equation (T + sigma) t = r gets one
multigrid cycle plus a network correction; the network is trained on the device, on residual
bands that the plain solver (multigrid preconditioner) produces, with targets from refined
multigrid cycles.  The unchanged residual test decides convergence, so the eigenvalues must not
change; the network must beat the single cycle on held-out residual bands.
"""
import math
import time

import numpy as np
import pytest

import dft_b200

pytestmark = pytest.mark.gpu


def _h2o(n, h):
    half = 0.5 * h * (n - 1)
    g = dft_b200.CartesianGrid(n, n, n, -half, half, -half, half, -half, half)
    ang = math.radians(104.5 / 2)
    Z = [8, 1, 1]
    xyz = np.array([0.013, 0.021, 0.017, 1.81 * math.sin(ang), 0.021, 1.81 * math.cos(ang),
                    -1.81 * math.sin(ang), 0.021, 1.81 * math.cos(ang)])
    return g, Z, xyz


def test_learned_preconditioner_trains_and_keeps_eigenvalues(engine):
    g, Z, xyz = _h2o(40, 0.3)
    N = g.getSize()
    V = engine.array(N)
    engine.nuclear_potential(g, Z, xyz, V)
    net = dft_b200.PoissonNet(engine, seed=11)
    rep = net.train_preconditioner(g, V, nocc=5, nbands=8, samples=64, validation=12, epochs=8, cycles=12)
    print("learned preconditioner: val loss", rep["val_loss"], "one cycle alone", rep["val_loss_coarse"],
          "train s", rep["seconds_train"])
    assert np.isfinite(rep["val_loss"]) and rep["val_loss"] < rep["val_loss_coarse"]
    res = {}
    for pc in (-1, -3):
        psi = engine.array(8 * N)
        t0 = time.perf_counter()
        eig, it = engine.solve_orbitals(g, V, 5, 8, psi, N, init=False, preconditioner=pc,
                                        preconditioner_net=net if pc == -3 else None)
        res[pc] = (eig, it, time.perf_counter() - t0)
    print("iterations multigrid", res[-1][1], "learned", res[-3][1], "seconds", res[-1][2], res[-3][2])
    assert np.max(np.abs(res[-3][0][:5] - res[-1][0][:5])) < 1e-9


def test_learned_preconditioner_needs_a_network(engine):
    g, Z, xyz = _h2o(16, 0.5)
    N = g.getSize()
    V = engine.array(N)
    engine.nuclear_potential(g, Z, xyz, V)
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.solve_orbitals(g, V, 5, 8, engine.array(8 * N), N, preconditioner=-3)
    assert ei.value.status == dft_b200.DFT_INVALID_ARGUMENT
