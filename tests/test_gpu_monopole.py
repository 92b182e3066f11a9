"""GPU: the monopole Hartree boundary (dft_scf_opts.hartree_boundary = 1, dft_hartree_monopole_dev).

The reference's faces carry Q/|r| only where a face's last node misses the bound by rounding
(HartreePotentialMolecule.cpp:45-94), so on the benchmark grids they are all zero.  The option
puts Q/|r| on every face; the solve goes through a Gaussian compensation charge and the
zero-face Jacobi sweeps.  The check is a direct sparse solve of the same 7-point Dirichlet
problem on the CPU.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import dft_b200

pytestmark = pytest.mark.gpu


def _axes(n, b):
    return [b[2 * d] + np.arange(n[d]) * ((b[2 * d + 1] - b[2 * d]) / (n[d] - 1)) for d in range(3)]


def _direct_monopole(n, b, rho):
    """Solve lap_h V = -4 pi rho on the interior with V = Q/|r| on every face (x fastest)."""
    nx, ny, nz = n
    x, y, z = _axes(n, b)
    h = [x[1] - x[0], y[1] - y[0], z[1] - z[0]]
    Zc, Yc, Xc = np.meshgrid(z, y, x, indexing="ij")
    dV = h[0] * h[1] * h[2]
    Q = rho.sum() * dV
    V = Q / np.sqrt(Xc ** 2 + Yc ** 2 + Zc ** 2)
    R = rho.reshape(nz, ny, nx)
    mi, mj, mk = nx - 2, ny - 2, nz - 2

    def lap1(m, hh):
        return sp.diags([np.ones(m - 1), -2 * np.ones(m), np.ones(m - 1)], [-1, 0, 1]) / hh ** 2

    A = (sp.kron(sp.kron(sp.identity(mk), sp.identity(mj)), lap1(mi, h[0]))
         + sp.kron(sp.kron(sp.identity(mk), lap1(mj, h[1])), sp.identity(mi))
         + sp.kron(sp.kron(lap1(mk, h[2]), sp.identity(mj)), sp.identity(mi)))
    Vb = V.copy()
    Vb[1:-1, 1:-1, 1:-1] = 0.0
    bound = np.zeros((mk, mj, mi))
    bound += (Vb[1:-1, 1:-1, :-2] + Vb[1:-1, 1:-1, 2:]) / h[0] ** 2
    bound += (Vb[1:-1, :-2, 1:-1] + Vb[1:-1, 2:, 1:-1]) / h[1] ** 2
    bound += (Vb[:-2, 1:-1, 1:-1] + Vb[2:, 1:-1, 1:-1]) / h[2] ** 2
    rhs = -4 * np.pi * R[1:-1, 1:-1, 1:-1] - bound
    V[1:-1, 1:-1, 1:-1] = spla.spsolve(A.tocsc(), rhs.ravel()).reshape(mk, mj, mi)
    return V.ravel(), Q


def _density(n, b, seed):
    rng = np.random.default_rng(seed)
    x, y, z = _axes(n, b)
    Zc, Yc, Xc = np.meshgrid(z, y, x, indexing="ij")
    rho = np.zeros(Xc.shape)
    for _ in range(3):
        c = rng.uniform(-1.5, 1.5, 3)
        rho += rng.uniform(0.3, 1.0) * np.exp(-((Xc - c[0]) ** 2 + (Yc - c[1]) ** 2 + (Zc - c[2]) ** 2) / 0.8)
    return rho.ravel()


# an exact-face grid (the reference would put 0 on every face) and a skewed one whose last
# nodes miss the bounds by rounding
@pytest.mark.parametrize("n,b", [((24, 24, 24), (-5.75, 5.75) * 3),
                                 ((23, 21, 19), (-5.3, 6.1, -4.9, 5.2, -4.4, 4.7))])
def test_monopole_matches_direct_solve(engine, n, b):
    g = dft_b200.CartesianGrid(*n, *b)
    rho = _density(n, b, 3)
    ref, Q = _direct_monopole(n, b, rho)
    d_rho, d_v = engine.upload(rho), engine.array(g.getSize())
    sweeps, last = engine.hartree_monopole(g, d_rho, d_v, tol=1e-13, max_sweeps=200000)
    v = d_v.to_host()
    assert last < 1e-13 and sweeps < 200000
    face = np.ones((n[2], n[1], n[0]), bool)
    face[1:-1, 1:-1, 1:-1] = False
    face = face.ravel()
    # faces: Q/|r| to rounding (the compensation's erf is 1 to double precision there)
    assert np.max(np.abs(v[face] - ref[face]) / np.abs(ref[face])) < 1e-13
    # interior: the Jacobi fixed point at tol 1e-13 is within ~1e-10 of the exact solution
    assert np.max(np.abs(v - ref)) < 1e-9 * max(1.0, abs(Q)), np.max(np.abs(v - ref))


def test_monopole_origin_outside_rejected(engine):
    g = dft_b200.CartesianGrid(16, 16, 16, 0.5, 8.0, -4.0, 4.0, -4.0, 4.0)
    d_rho, d_v = engine.upload(np.zeros(g.getSize())), engine.array(g.getSize())
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.hartree_monopole(g, d_rho, d_v)
    assert ei.value.status == dft_b200.DFT_INVALID_ARGUMENT


def _h2():
    m = dft_b200.Molecule()
    m.addNucleus(1, -0.7, 0, 0)
    m.addNucleus(1, 0.7, 0, 0)
    return m


def test_scf_monopole_boundary(engine):
    """The option reaches the |dE| stop; Q/|r| > 0 on the faces raises V_H everywhere (maximum principle),
    so the occupied level sits above the zero-face one.  An unknown value is rejected."""
    g = dft_b200.CartesianGrid(40, 40, 40, -7.8, 7.8, -7.8, 7.8, -7.8, 7.8)
    base = dict(poisson_start=5, mixer=1, adaptive_eig_tol=1, stop_abs_de=1e-6)
    r0 = engine.scf_molecule(g, _h2(), 0, 1, "PZ81", dft_b200.default_scf_options(**base))
    r1 = engine.scf_molecule(g, _h2(), 0, 1, "PZ81", dft_b200.default_scf_options(hartree_boundary=1, **base))
    assert r0.energyDifference < 1e-6 and r1.energyDifference < 1e-6  # the stop_abs_de test ended both
    assert r1.eigenvalues[0] > r0.eigenvalues[0] + 0.05
    assert r1.energy.hartree > r0.energy.hartree
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.scf_molecule(g, _h2(), 0, 1, "PZ81", dft_b200.default_scf_options(hartree_boundary=2, max_iterations=1))
    assert ei.value.status == dft_b200.DFT_INVALID_ARGUMENT


def test_scf_monopole_with_hartree_start_from_mixer(engine):
    """With the monopole boundary the Hartree start from the mixer is combined from potentials
    whose total charges differ by rounding and clamping; its faces are zeroed before the
    zero-face multigrid, so every Jacobi finish stays short (it ran into the 10,000-sweep cap
    before) and the energy equals the previous-potential start's."""
    g = dft_b200.CartesianGrid(40, 40, 40, -7.8, 7.8, -7.8, 7.8, -7.8, 7.8)
    base = dict(poisson_start=5, mixer=1, adaptive_eig_tol=1, stop_abs_de=1e-8, stop_abs_deig=1e-8,
                hartree_boundary=1)
    r0 = engine.scf_molecule(g, _h2(), 0, 1, "PZ81", dft_b200.default_scf_options(**base))
    r1 = engine.scf_molecule(g, _h2(), 0, 1, "PZ81", dft_b200.default_scf_options(poisson_predict=1, **base))
    assert max(h["poisson_sweeps_in"] for h in r1.history) < 100, [h["poisson_sweeps_in"] for h in r1.history]
    assert abs(r1.total - r0.total) < 1e-7
