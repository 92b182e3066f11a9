"""GPU: failure paths end in a status code, never in a hang or a fault.

Each failure is made on the host: a tuning key that shortens a bounded device wait or
tightens a pivot test, or a NaN placed in an input.  The device code only takes its normal
give-up branch; the context stays usable afterwards.  References: the singular Thomas pivot
(NumericalMethods.cpp:105-122), the Davidson's non-finite guards
(EigenvalueSolverMolecule.cpp:1214-1220).
"""
import numpy as np
import pytest

import dft_b200
from conftest import gaussian_density

pytestmark = pytest.mark.gpu


def test_persistent_jacobi_barrier_gives_up(engine):
    """With a grid-barrier poll limit of 1 the persistent Jacobi launch gives up at its first
    barrier: DFT_CUDA_ERROR with a message, then the same context solves normally."""
    n, b = (64, 64, 64), (-6.3, 6.3) * 3
    g = dft_b200.CartesianGrid(*n, *b)
    na, nb = gaussian_density(n, b, 3)
    rho = na + nb
    d_rho, d_vh = engine.upload(rho), engine.array(rho.size)
    engine.set_tuning("jacobi_sweeps_per_launch", -1)
    try:
        engine.set_tuning("grid_barrier_poll_limit", 1)
        with pytest.raises(dft_b200.DFTError) as ei:
            engine.hartree(g, d_rho, d_vh, 1e-8, 10000)
        assert ei.value.status == dft_b200.DFT_CUDA_ERROR
        assert "timed out" in str(ei.value)
        engine.set_tuning("grid_barrier_poll_limit", 0)
        sweeps, _ = engine.hartree(g, d_rho, d_vh, 1e-8, 300)
        assert sweeps == 300
        engine.set_tuning("jacobi_sweeps_per_launch", 1)
        d_ref = engine.array(rho.size)
        engine.hartree(g, d_rho, d_ref, 1e-8, 300)
        assert np.array_equal(d_vh.to_host(), d_ref.to_host())
    finally:
        engine.set_tuning("grid_barrier_poll_limit", 0)
        engine.set_tuning("jacobi_sweeps_per_launch", 0)


def test_nan_in_potential_is_numerical(engine):
    """A NaN in the effective potential ends the eigensolver with DFT_NUMERICAL."""
    n, b = (16, 16, 16), (-6.0, 6.0) * 3
    g = dft_b200.CartesianGrid(*n, *b)
    N = g.getSize()
    V = -1.0 / (1.0 + np.arange(N) % 7)
    V[N // 2 + 3] = np.nan
    psi = engine.array(4 * N)
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.solve_orbitals(g, engine.upload(V), 2, 4, psi, N, init=False)
    assert ei.value.status == dft_b200.DFT_NUMERICAL
    # the context still works
    V[N // 2 + 3] = -0.5
    eig, _ = engine.solve_orbitals(g, engine.upload(V), 2, 4, psi, N, init=False)
    assert np.all(np.isfinite(eig))


def test_singular_radial_pivot(engine):
    """A pivot tolerance no pivot can meet makes every run report DFT_SINGULAR, without
    stopping the other runs' launch; the default tolerance then reproduces the normal runs."""
    try:
        engine.set_tuning("radial_pivot_exponent", 300)
        res = engine.solve_atoms([1, 6], ["PZ81", "PBE96"])
        assert [r.status for r in res] == [dft_b200.DFT_SINGULAR] * 2
    finally:
        engine.set_tuning("radial_pivot_exponent", -14)
    res = engine.solve_atoms([1, 6], ["PZ81", "PBE96"])
    assert [r.status for r in res] == [dft_b200.DFT_OK] * 2
    assert abs(res[0].energy.total - (-0.478407096)) < 5e-8
