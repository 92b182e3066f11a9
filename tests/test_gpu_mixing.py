"""GPU: the Kerker-screened density mixers and the multigrid cycle they rest on.

Kerker screening (dft_scf_opts.kerker_q0) multiplies the total-charge residual by
-lap/(-lap + q0^2), computed with one multigrid V-cycle for the screened Poisson equation.
The reference mixes linearly (MolecularSCFHelpers.cpp:27-44); these are options, and the
unchanged SCF stop tests decide convergence, so the energies must match the linear mixer's.
"""
import numpy as np
import pytest

import dft_b200

pytestmark = pytest.mark.gpu


def _neg_lap_plus(n, b, x, q2):
    """(-lap_h + q2) x with the 7-point stencil, x = 0 outside the box (x fastest)."""
    nx, ny, nz = n
    h = [(b[1] - b[0]) / (nx - 1), (b[3] - b[2]) / (ny - 1), (b[5] - b[4]) / (nz - 1)]
    X = x.reshape(nz, ny, nx)
    P = np.pad(X, 1)
    out = (2 * sum(1 / hh ** 2 for hh in h) + q2) * X
    out -= (P[1:-1, 1:-1, 2:] + P[1:-1, 1:-1, :-2]) / h[0] ** 2
    out -= (P[1:-1, 2:, 1:-1] + P[1:-1, :-2, 1:-1]) / h[1] ** 2
    out -= (P[2:, 1:-1, 1:-1] + P[:-2, 1:-1, 1:-1]) / h[2] ** 2
    return out.ravel()


@pytest.mark.parametrize("n,b", [((64, 64, 64), (-6.3, 6.3) * 3), ((45, 38, 33), (-5.0, 5.0, -4.2, 4.2, -3.6, 3.6))])
@pytest.mark.parametrize("q2", [0.25, 1.0])
@pytest.mark.parametrize("cycles,bar", [(1, 0.5), (2, 0.35)])
def test_screened_poisson_cycle_contracts(engine, n, b, q2, cycles, bar):
    """One V-cycle from zero removes more than half of the residual of (-lap + q2) x = src, two
    (the Kerker mixer's setting) about three quarters (0.27 measured on the 45 x 38 x 33 grid,
    whose coarse levels do not nest), and the map is linear (doubling the source doubles x
    exactly)."""
    g = dft_b200.CartesianGrid(*n, *b)
    N = g.getSize()
    rng = np.random.default_rng(5)
    x0, y0, z0 = [np.linspace(b[2 * d], b[2 * d + 1], n[d]) for d in range(3)]
    Zc, Yc, Xc = np.meshgrid(z0, y0, x0, indexing="ij")
    src = np.zeros(N)
    for _ in range(6):  # smooth charges of both signs plus grid-scale noise
        c = rng.uniform(-2, 2, 3)
        src += rng.uniform(-1, 1) * np.exp(-((Xc - c[0]) ** 2 + (Yc - c[1]) ** 2 + (Zc - c[2]) ** 2)).ravel()
    src += 0.05 * rng.standard_normal(N)
    d_src, d_x = engine.upload(src), engine.array(N)
    engine.screened_poisson(g, d_src, d_x, q2, cycles)
    x = d_x.to_host()
    r = src - _neg_lap_plus(n, b, x, q2)
    assert np.linalg.norm(r) < bar * np.linalg.norm(src), np.linalg.norm(r) / np.linalg.norm(src)
    d2, x2 = engine.upload(2.0 * src), engine.array(N)
    engine.screened_poisson(g, d2, x2, q2, cycles)
    assert np.array_equal(x2.to_host(), 2.0 * x)


@pytest.mark.parametrize("case", ["h2_closed", "h3_doublet"])
def test_kerker_mixers_same_energy(engine, case):
    """Pulay + Kerker and linear + Kerker reach the linear mixer's energy (the stop tests
    are unchanged), closed and open shell."""
    g = dft_b200.CartesianGrid(28, 28, 28, -5.4, 5.4, -5.4, 5.4, -5.4, 5.4)
    m = dft_b200.Molecule()
    if case == "h2_closed":
        m.addNucleus(1, -0.7, 0.0, 0.0)
        m.addNucleus(1, 0.7, 0.0, 0.0)
        mult = 1
    else:
        m.addNucleus(1, -1.6, 0.0, 0.0)
        m.addNucleus(1, 0.0, 0.1, 0.0)
        m.addNucleus(1, 1.6, 0.0, 0.0)
        mult = 2
    res = {}
    for mixer, q0 in ((0, 0.0), (1, 0.8), (0, 0.8)):
        o = dft_b200.default_scf_options(stop_abs_de=1e-8, poisson_start=dft_b200.POISSON_MULTIGRID, mixer=mixer,
                                         kerker_q0=q0)
        r = engine.scf_molecule(g, m, 0, mult, "PBE96", o)
        res[(mixer, q0)] = (r.total, r.iterations)
    print(case, res)
    e0 = res[(0, 0.0)][0]
    for k, (e, it) in res.items():
        assert abs(e - e0) < 1e-6, (k, res)


def test_kerker_rejects_negative_q0(engine):
    g = dft_b200.CartesianGrid(12, 12, 12, -3.0, 3.0, -3.0, 3.0, -3.0, 3.0)
    m = dft_b200.Molecule()
    m.addNucleus(1, -0.7, 0.05, 0.0)
    m.addNucleus(1, 0.7, 0.05, 0.0)
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.scf_molecule(g, m, 0, 1, "PZ81", dft_b200.default_scf_options(kerker_q0=-1.0))
    assert ei.value.status == dft_b200.DFT_INVALID_ARGUMENT


@pytest.mark.parametrize("mixer,q0,mult", [(1, 0.0, 1), (0, 0.0, 1), (1, 0.8, 1), (1, 0.0, 2)])
def test_poisson_predict_same_energy_fewer_cycles(engine, mixer, q0, mult):
    """The mixer's own V_H combination as the start of each V_H(n_in) solve (poisson_predict 1,
    and 2 with the V_H(n_out) start as well) ends at the same Jacobi stop rule: the same energy
    as the previous-potential start, with fewer multigrid cycles for n_in after the first
    iterations (Pulay, linear, Pulay + Kerker, open shell)."""
    g = dft_b200.CartesianGrid(32, 32, 32, -6.2, 6.2, -6.2, 6.2, -6.2, 6.2)
    m = dft_b200.Molecule()
    if mult == 1:
        m.addNucleus(1, -0.7, 0.0, 0.0)
        m.addNucleus(1, 0.7, 0.0, 0.0)
    else:
        m.addNucleus(1, -1.6, 0.0, 0.0)
        m.addNucleus(1, 0.0, 0.1, 0.0)
        m.addNucleus(1, 1.6, 0.0, 0.0)
    res = {}
    for pp in (0, 1, 2):
        o = dft_b200.default_scf_options(stop_abs_de=1e-8, stop_abs_deig=1e-8,
                                         poisson_start=dft_b200.POISSON_MULTIGRID, mixer=mixer, kerker_q0=q0,
                                         poisson_predict=pp)
        r = engine.scf_molecule(g, m, 0, mult, "PBE96", o)
        assert r.converged or r.energyDifference < 1e-8
        res[pp] = (r.total, [h["poisson_cycles_in"] for h in r.history], r.eigenvalues,
                   [h["poisson_cycles_out"] for h in r.history])
    print(mixer, q0, mult, res)
    for pp in (1, 2):
        assert abs(res[pp][0] - res[0][0]) < 1e-7
        assert np.max(np.abs(np.subtract(res[pp][2], res[0][2]))) < 1e-6
        n = min(len(res[0][1]), len(res[pp][1]))
        assert sum(res[pp][1][2:n]) < 0.7 * sum(res[0][1][2:n]), res


def test_poisson_predict_rejects_unknown(engine):
    g = dft_b200.CartesianGrid(12, 12, 12, -3.0, 3.0, -3.0, 3.0, -3.0, 3.0)
    m = dft_b200.Molecule()
    m.addNucleus(1, -0.7, 0.05, 0.0)
    m.addNucleus(1, 0.7, 0.05, 0.0)
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.scf_molecule(g, m, 0, 1, "PZ81", dft_b200.default_scf_options(poisson_predict=3, max_iterations=1))
    assert ei.value.status == dft_b200.DFT_INVALID_ARGUMENT
