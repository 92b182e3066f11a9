"""GPU: the superposed-radial-atoms start of the molecular SCF (dft_scf_opts.initial_density = 1).

The reference starts from orbitals of the bare nuclear potential
(buildInitialMolecularDensities, MolecularSCFHelpers.cpp:515-579).  The option starts from
the batched radial atoms (SelfConsistentField.cpp:539-786) instead; the SCF stop tests are
unchanged, so the converged energy and eigenvalues must be the same (the SCF iteration counts
are printed: the start saves the bare-potential eigensolve, not necessarily SCF iterations).
"""
import math

import numpy as np
import pytest

import dft_b200

pytestmark = pytest.mark.gpu


def _h2o(n=32, h=0.3):
    half = 0.5 * h * (n - 1)
    g = dft_b200.CartesianGrid(n, n, n, -half, half, -half, half, -half, half)
    ang = math.radians(104.5 / 2)
    m = dft_b200.Molecule()
    m.addNucleus(8, 0.013, 0.021, 0.017)
    m.addNucleus(1, 1.81 * math.sin(ang), 0.021, 1.81 * math.cos(ang))
    m.addNucleus(1, -1.81 * math.sin(ang), 0.021, 1.81 * math.cos(ang))
    return g, m


@pytest.mark.parametrize("case", ["h2o_closed", "nh_triplet", "h3_doublet"])
def test_atomic_start_same_energy(engine, case):
    if case == "h2o_closed":
        g, m = _h2o()
        mult, fn = 1, "PBE96"
    elif case == "nh_triplet":
        g, _ = _h2o()
        m = dft_b200.Molecule()
        m.addNucleus(7, 0.013, 0.021, 0.017)
        m.addNucleus(1, 1.96, 0.021, 0.017)
        mult, fn = 3, "PZ81"
    else:
        g = dft_b200.CartesianGrid(28, 28, 28, -5.4, 5.4, -5.4, 5.4, -5.4, 5.4)
        m = dft_b200.Molecule()
        m.addNucleus(1, -1.6, 0.0, 0.0)
        m.addNucleus(1, 0.0, 0.1, 0.0)
        m.addNucleus(1, 1.6, 0.0, 0.0)
        mult, fn = 2, "PBE96"
    res = {}
    for start in (0, 1):
        o = dft_b200.default_scf_options(stop_abs_de=1e-8, poisson_start=dft_b200.POISSON_MULTIGRID, mixer=1,
                                         eig_preconditioner=-1, initial_density=start)
        r = engine.scf_molecule(g, m, 0, mult, fn, o)
        res[start] = (r.total, r.iterations, r.eigenvalues)
    print(case, {k: v[:2] for k, v in res.items()})
    assert abs(res[1][0] - res[0][0]) < 1e-6, res
    assert np.max(np.abs(np.array(res[1][2]) - np.array(res[0][2]))) < 1e-5


def test_atomic_start_rejects_heavy_elements(engine):
    g = dft_b200.CartesianGrid(16, 16, 16, -4.0, 4.0, -4.0, 4.0, -4.0, 4.0)
    m = dft_b200.Molecule()
    m.addNucleus(31, 0.01, 0.02, 0.03)
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.scf_molecule(g, m, 0, 2, "PZ81", dft_b200.default_scf_options(initial_density=1, max_iterations=1))
    assert ei.value.status == dft_b200.DFT_INVALID_ARGUMENT
