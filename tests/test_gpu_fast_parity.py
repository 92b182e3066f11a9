"""GPU: the fast configuration against an FP64 oracle run of the plain method.

The fast configuration (multigrid Poisson starts taken to the Jacobi fixed point, the Hartree
start from the mixer, mixed-precision eigensolver with its multigrid preconditioner, Pulay
mixing, adaptive eigensolver tolerance, stop at
|dE| < 1e-7 Ha with every occupied eigenvalue changed by < 1e-7 Ha and dRho < 5e-7, the bench's
stop) must agree with the plain method run to its fixed point in FP64: the
reference's linear mixer and FP64 eigensolver, each Poisson solve stopped where its
iterate is within ~1e-8 of the Jacobi fixed point (the reference's max|dV| < 1e-8 rule
scaled by 1 - rho_Jacobi; the multigrid start only shortens the way there), SCF to
|dE| < 1e-9.  Bar: |E_tot - E_oracle| <= 1e-6 Ha and every occupied eigenvalue within
1e-6 Ha (reference loop: MolecularSCFIteration.cpp:12-252).
"""
import math

import numpy as np
import pytest

import dft_b200
from dft_b200 import systems

pytestmark = pytest.mark.gpu


def _tight_tol(n, b, tol=1e-8):
    d = [(b[2 * i + 1] - b[2 * i]) / (n[i] - 1) for i in range(3)]
    inv = [1.0 / (x * x) for x in d]
    rho = sum(c * math.cos(math.pi / (m - 1)) for c, m in zip(inv, n)) / sum(inv)
    return tol * (1.0 - rho)


def _h2o_64():
    n, h = 64, 0.3
    half = 0.5 * h * (n - 1)
    ang = math.radians(104.5 / 2)
    # 5 occupied + 27 buffer bands: the basis (3 x 32) x 32 products run on the tensor cores
    return dict(n=(n, n, n), bounds=(-half, half) * 3, Z=[8, 1, 1],
                xyz=[[0.011, 0.017, 0.023], [1.81 * math.sin(ang), 0.017, 1.81 * math.cos(ang)],
                     [-1.81 * math.sin(ang), 0.017, 1.81 * math.cos(ang)]],
                multiplicity=1, functional="PBE96", extra_bands=27)


@pytest.mark.parametrize("name", ["h2_48", "h2o_64"])
def test_fast_configuration_matches_fp64_oracle(engine, name):
    w = systems.h2_48() if name == "h2_48" else _h2o_64()
    g = dft_b200.CartesianGrid(*w["n"], *w["bounds"])
    m = dft_b200.Molecule()
    for z, p in zip(w["Z"], w["xyz"]):
        m.addNucleus(z, *p)
    oracle = dft_b200.default_scf_options(stop_abs_de=1e-9, stop_abs_deig=1e-9, extra_bands=w["extra_bands"],
                                         poisson_start=dft_b200.POISSON_MULTIGRID,
                                         poisson_tol=_tight_tol(w["n"], w["bounds"]), poisson_max_sweeps=400000,
                                         eig_preconditioner=-1)
    fast = dft_b200.default_scf_options(stop_abs_de=1e-7, stop_abs_deig=1e-7, stop_abs_drho=5e-7,
                                        extra_bands=w["extra_bands"],
                                        poisson_start=dft_b200.POISSON_MULTIGRID, eig_mixed_precision=1,
                                        eig_preconditioner=-2, mixer=1, adaptive_eig_tol=1, poisson_predict=1,
                                        poisson_fixed_point=1)
    ro = engine.scf_molecule(g, m, 0, w["multiplicity"], w["functional"], oracle)
    tc0 = engine.counter("tensor_core_products")
    rf = engine.scf_molecule(g, m, 0, w["multiplicity"], w["functional"], fast)
    tc = engine.counter("tensor_core_products") - tc0
    de = rf.total - ro.total
    deig = np.max(np.abs(np.array(rf.eigenvalues) - np.array(ro.eigenvalues)))
    print(name, "E fast", rf.total, "oracle", ro.total, "dE", de, "max deig", deig, "iterations", rf.iterations,
          ro.iterations, "tensor-core products", tc)
    assert abs(de) <= 1e-6
    assert deig <= 1e-6
    if name == "h2o_64":
        assert tc > 0, "the mixed-precision products did not reach the tensor cores"
