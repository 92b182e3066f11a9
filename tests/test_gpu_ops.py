"""GPU parity of the 3D operators against the CPU oracle (oracle/dft_oracle.c, itself pinned
bit-for-bit to the reference in test_oracle_pin.py) and the reference's own fixture.

Bars: H psi, Jacobi Poisson (values and sweep count), density and the nuclear potential are
bit-identical; XC and reductions agree to relative 1e-12 (device libm and summation order).
"""
import numpy as np
import pytest

import dft_b200
from conftest import gaussian_density, golden, grid_coords
from oracle.bindings import PBE96, PZ81

pytestmark = pytest.mark.gpu

GRIDS = [
    ((11, 9, 8), (-3.0, 3.4, -2.5, 2.9, -2.2, 2.0)),
    ((33, 17, 21), (-4.0, 4.0, -2.0, 2.0, -2.5, 2.5)),
    ((5, 6, 4), (-2.0, 2.2, -1.0, 1.5, -1.7, 1.3)),   # faces not exactly on xmax: non-zero boundary values
    ((48, 48, 48), (-7.05, 7.05) * 3),                 # the H2 48^3, h = 0.3 grid
]
XC_RTOL = 1e-12


def G(n, b):
    return dft_b200.CartesianGrid(*n, *b)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(params=[(0, 0), (0, 1), (0, 2), (0, 4), (1, 1), (1, 2), (2, 0), (2, 8), (3, 0)],
                ids=lambda t: f"v{t[0]}bpt{t[1]}")
def hpsi_bands_per_thread(request, engine):
    """Every H psi launch shape: neighbours through L1 (variant 0) with auto, 1, 2 or 4 bands per
    thread, the shared-memory plane tile (variant 1) with 1 or 2, and the TMA plane ring
    (variant 2, 4 or 8 bands per block; an odd leading dimension falls back to variant 0) and the
    prefetching single-band march (variant 3)."""
    variant, bpt = request.param
    engine.set_tuning("hpsi_variant", variant)
    engine.set_tuning("hpsi_bands_per_thread", bpt)
    yield request.param
    engine.set_tuning("hpsi_bands_per_thread", 0)
    engine.set_tuning("hpsi_variant", 0)


@pytest.mark.parametrize("n,b", [((12, 9, 8), (-3.0, 3.4, -2.5, 2.9, -2.2, 2.0)),
                                 ((34, 17, 21), (-4.0, 4.0, -2.0, 2.0, -2.5, 2.5)),
                                 ((6, 6, 4), (-2.0, 2.2, -1.0, 1.5, -1.7, 1.3)),
                                 ((70, 41, 37), (-7.0, 7.0, -4.0, 4.0, -3.6, 3.6)),
                                 ((48, 48, 48), (-7.05, 7.05) * 3)])
@pytest.mark.parametrize("nbc", [0, 1, 2, 8])
def test_hpsi_tma_ring_bit_exact(engine, port, n, b, nbc):
    """The TMA plane ring (hpsi_variant 2): even nx and ld, tiles that overhang the grid in x and
    y, several z-chunks, band runs of 1, 2, 4 (auto) and 8 with a partial last run; every value
    bit for bit (signed zeros included) against the oracle."""
    rng = np.random.default_rng(12)
    N = int(np.prod(n))
    nb_, ld = 7, N + 38
    V = rng.standard_normal(N)
    psi = np.zeros((nb_, ld))
    psi[:, :N] = rng.standard_normal((nb_, N))
    psi[2, : N // 3] = 0.0  # runs of zeros: the skipped-neighbour order decides the sign of zero
    dV, dP, dH = engine.upload(V), engine.upload(psi), engine.array(nb_ * ld)
    engine.set_tuning("hpsi_variant", 2)
    engine.set_tuning("hpsi_bands_per_thread", nbc)
    try:
        engine.apply_hamiltonian(G(n, b), dV, dP, dH, nb_, ld)
        engine.synchronize()
    finally:
        engine.set_tuning("hpsi_bands_per_thread", 0)
        engine.set_tuning("hpsi_variant", 0)
    H = dH.to_host((nb_, ld))
    for k in range(nb_):
        assert H[k, :N].tobytes() == port.apply_hamiltonian(n, b, V, psi[k, :N]).tobytes(), k


@pytest.mark.parametrize("n,b", GRIDS)
def test_hpsi_bit_exact(engine, port, n, b, hpsi_bands_per_thread):
    rng = np.random.default_rng(11)
    N = int(np.prod(n))
    nb_, ld = 5, N + 37  # padded leading dimension; 5 bands leave a partial group of 2 or 4
    V = rng.standard_normal(N)
    psi = np.zeros((nb_, ld))
    psi[:, :N] = rng.standard_normal((nb_, N))
    dV, dP, dH = engine.upload(V), engine.upload(psi), engine.array(nb_ * ld)
    engine.apply_hamiltonian(G(n, b), dV, dP, dH, nb_, ld)
    H = dH.to_host((nb_, ld))
    for k in range(nb_):
        assert np.array_equal(H[k, :N], port.apply_hamiltonian(n, b, V, psi[k, :N])), k


def test_hpsi_large_numpy_restatement(engine, hpsi_bands_per_thread):
    """128^3 x 4 bands: bit-identical to a vectorised numpy restatement of the same stencil order."""
    n, b = (128, 128, 128), (-12.7, 12.7) * 3
    g = G(n, b)
    N = g.getSize()
    rng = np.random.default_rng(5)
    V = rng.standard_normal(N)
    psi = rng.standard_normal((4, N))
    dH = engine.array(4 * N)
    engine.apply_hamiltonian(g, engine.upload(V), engine.upload(psi), dH, 4, N)
    H = dH.to_host((4, N))
    dx = (b[1] - b[0]) / (n[0] - 1)
    ix = 1.0 / (dx * dx)
    k0 = -2.0 * (ix + ix + ix)
    for band in (0, 3):
        p = psi[band].reshape(n[2], n[1], n[0])
        lap = k0 * p
        for ax, sl in ((2, -1), (2, 1), (1, -1), (1, 1), (0, -1), (0, 1)):
            nb = np.zeros_like(p)
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            if sl == -1:  # neighbour at index-1
                dst[ax], src[ax] = slice(1, None), slice(None, -1)
            else:
                dst[ax], src[ax] = slice(None, -1), slice(1, None)
            nb[tuple(dst)] = p[tuple(src)] * ix
            mask = np.zeros_like(p, dtype=bool)
            mask[tuple(dst)] = True
            lap = np.where(mask, lap + nb, lap)
        ref = -0.5 * lap + V.reshape(p.shape) * p
        assert np.array_equal(H[band], ref.ravel())


@pytest.fixture(params=[0, -2, -1, 1, 2, 4, 8], ids=lambda t: f"spl{t}")
def sweeps_per_launch(request, engine):
    """Every Jacobi launch shape: auto, cluster-resident (-2), persistent (-1), one sweep per
    launch (1), temporal blocks of 2/4/8."""
    engine.set_tuning("jacobi_sweeps_per_launch", request.param)
    yield request.param
    engine.set_tuning("jacobi_sweeps_per_launch", 0)


@pytest.mark.parametrize("n,b", GRIDS + [((24, 24, 24), (-6.0, 6.0) * 3), ((40, 37, 70), (-6.0, 6.0) * 3),
                                         ((33, 31, 35), (-6.0, 6.1, -6.0, 5.9, -5.5, 6.2))])
def test_jacobi_bit_exact_and_sweeps(engine, port, n, b, sweeps_per_launch):
    if sweeps_per_launch == -2 and n[2] < 32:
        pytest.skip("the cluster-resident solver needs nz >= 32")
    na, nb = gaussian_density(n, b, 2)
    rho = na + nb
    ref = np.empty(rho.size)
    import ctypes as C
    sw = C.c_long()
    ld = C.c_double()
    port.check(port.fn("hartree_potential_ex")(np.asarray(n, dtype=np.int64).ctypes.data_as(C.POINTER(C.c_long)),
                                               np.asarray(b, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                               rho.ctypes.data_as(C.POINTER(C.c_double)),
                                               ref.ctypes.data_as(C.POINTER(C.c_double)), C.byref(sw), C.byref(ld)))
    d_rho, d_vh = engine.upload(rho), engine.array(rho.size)
    sweeps, last = engine.hartree(G(n, b), d_rho, d_vh)
    assert sweeps == sw.value
    assert last == ld.value
    assert np.array_equal(d_vh.to_host(), ref)


def test_jacobi_cap(engine, port, sweeps_per_launch):
    """The silent sweep cap (HartreePotentialMolecule.cpp:207): stop after max_sweeps, with the
    iterate of exactly that sweep (37 is not a multiple of any block size)."""
    n, b = (24, 24, 40), (-6.0, 6.0) * 3
    na, nb = gaussian_density(n, b, 4)
    d_rho, d_vh = engine.upload(na + nb), engine.array(na.size)
    sweeps, last = engine.hartree(G(n, b), d_rho, d_vh, tol=1e-8, max_sweeps=37)
    assert sweeps == 37 and last > 1e-8
    v37 = d_vh.to_host()
    engine.set_tuning("jacobi_sweeps_per_launch", 1)
    ref = engine.array(na.size)
    engine.hartree(G(n, b), d_rho, ref, tol=1e-8, max_sweeps=37)
    assert np.array_equal(v37, ref.to_host())
    engine.set_tuning("jacobi_sweeps_per_launch", sweeps_per_launch)
    sweeps0, _ = engine.hartree(G(n, b), d_rho, d_vh, tol=1e-8, max_sweeps=0)
    assert sweeps0 == 0


def test_reference_ops_fixture(engine):
    """Against outputs of the reference itself (tests/golden/ops_ref.json)."""
    fx = golden("ops_ref.json")
    n, b = tuple(fx["n"]), tuple(fx["bounds"])
    g = G(n, b)
    N = g.getSize()
    na, nb, V = map(np.asarray, (fx["na"], fx["nb"], fx["V"]))
    psi = np.asarray(fx["psi"])
    dH = engine.array(3 * N)
    engine.apply_hamiltonian(g, engine.upload(V), engine.upload(psi), dH, 3, N)
    assert np.array_equal(dH.to_host((3, N)), np.asarray(fx["hpsi"]))
    dvh = engine.array(N)
    engine.hartree(g, engine.upload(na + nb), dvh)
    assert np.array_equal(dvh.to_host(), np.asarray(fx["vh"]))
    d_na, d_nb = engine.upload(na), engine.upload(nb)
    for kind, tag in ((PZ81, "pz81"), (PBE96, "pbe96")):
        va, vb = engine.array(N), engine.array(N)
        exc = engine.xc(g, kind, d_na, d_nb, va, vb)
        assert rel(va.to_host(), fx[f"vxc_{tag}_a"]) < XC_RTOL
        assert rel(vb.to_host(), fx[f"vxc_{tag}_b"]) < XC_RTOL
        assert abs(exc - fx[f"exc_{tag}"]) <= XC_RTOL * abs(fx[f"exc_{tag}"])
    d_psi = engine.upload(psi)
    assert abs(engine.kinetic_energy(g, d_psi, 3, N, [1, 1, 1]) - fx["T"]) <= 1e-12 * abs(fx["T"])
    dd = engine.array(N)
    engine.spin_density(N, d_psi, 3, N, [1, 1, 1], dd)
    assert np.array_equal(dd.to_host(), np.asarray(fx["dens"]))
    dv = engine.array(N)
    engine.nuclear_potential(g, fx["Zs"], np.ravel(fx["xyz"]), dv)
    assert np.array_equal(dv.to_host(), np.asarray(fx["vext"]))


@pytest.mark.parametrize("n,b", GRIDS)
@pytest.mark.parametrize("kind", [PZ81, PBE96])
def test_xc_potential_and_energy(engine, port, n, b, kind):
    na, nb = gaussian_density(n, b, 9)
    g = G(n, b)
    N = g.getSize()
    va, vb = engine.array(N), engine.array(N)
    e = engine.xc(g, kind, engine.upload(na), engine.upload(nb), va, vb)
    assert rel(va.to_host(), port.xc_potential(kind, n, b, na, nb, 0)) < XC_RTOL
    assert rel(vb.to_host(), port.xc_potential(kind, n, b, na, nb, 1)) < XC_RTOL
    eo = port.xc_energy(kind, n, b, na, nb)
    assert abs(e - eo) <= XC_RTOL * abs(eo)


@pytest.mark.parametrize("kind", [PZ81, PBE96])
def test_xc_evaluate_pointwise(engine, port, kind):
    """Physical inputs: densities 1e-10..1e2 (plus floored and one-spin points) with reduced
    gradients s = |g| / (2 kF n) in [0, 10].  (At n ~ 1e-19 with O(1) gradients the PBE
    intermediates overflow in the reference as well; those points carry no meaning.)"""
    rng = np.random.default_rng(3)
    m = 20000
    na = 10.0 ** rng.uniform(-10, 2, m)
    nb = 10.0 ** rng.uniform(-10, 2, m)
    nb[::7] = 0.0
    na[::11] = 0.0
    na[::97] = 1e-21  # below the floor
    kfa = (3 * np.pi ** 2 * 2 * na) ** (1 / 3)
    kfb = (3 * np.pi ** 2 * 2 * nb) ** (1 / 3)
    ga = rng.uniform(-10, 10, m) * kfa * na
    gb = rng.uniform(-10, 10, m) * kfb * nb
    ga[::13] = 0.0
    out = engine.array(5 * m)
    engine.xc_evaluate(kind, m, engine.upload(na), engine.upload(nb), engine.upload(ga), engine.upload(gb), out)
    got = out.to_host((m, 5))
    want = port.xc_evaluate(kind, na, nb, ga, gb)
    # |got - want| <= 1e-10 |want| + 1e-13 max|column|: pointwise values pass through
    # cancellations (e.g. (1+z)^(4/3) + (1-z)^(4/3) - 2 near z = 0) where a last-ulp difference
    # of a transcendental is amplified; the grid-level potentials are held to 1e-12 above.
    colmax = np.max(np.abs(want), axis=0)
    bad = np.abs(got - want) > 1e-10 * np.abs(want) + 1e-13 * colmax
    if bad.any():
        i, c = np.argwhere(bad)[0]
        pytest.fail(f"point {i} column {c}: got {got[i, c]!r} want {want[i, c]!r} "
                    f"(na={na[i]!r} nb={nb[i]!r} ga={ga[i]!r} gb={gb[i]!r}); {bad.sum()} bad")


def test_density_kinetic_bit_and_tol(engine, port):
    n, b = (33, 17, 21), (-4.0, 4.0, -2.0, 2.0, -2.5, 2.5)
    g = G(n, b)
    N = g.getSize()
    rng = np.random.default_rng(8)
    psi = rng.standard_normal((5, N))
    occ = [1, 1, 0, 2, 1]
    d = engine.array(N)
    dp = engine.upload(psi)
    engine.spin_density(N, dp, 5, N, occ, d)
    assert np.array_equal(d.to_host(), port.spin_density(psi, occ))
    t = engine.kinetic_energy(g, dp, 5, N, occ)
    to = port.kinetic_energy(n, b, psi, occ)
    assert abs(t - to) <= 1e-12 * abs(to)


def test_nuclear_potential(engine, port):
    n, b = (48, 48, 48), (-7.05, 7.05) * 3
    Z = [8, 1, 1, 6]
    xyz = np.array([0.0, 0.01, 0.0, 1.4305, 0.0, 1.1084, -1.4305, 0.0, 1.1084, 2.0, 2.1, -1.3])
    d = engine.array(48 ** 3)
    engine.nuclear_potential(G(n, b), Z, xyz, d)
    assert np.array_equal(d.to_host(), port.nuclear_potential(n, b, Z, xyz))
    X, Y, Zc = grid_coords(n, b)
    on_node = [1, X[1000], Y[1000], Zc[1000]]
    with pytest.raises(dft_b200.DFTError) as ei:
        engine.nuclear_potential(G(n, b), [1], np.array(on_node[1:]), d)
    assert ei.value.status == dft_b200.DFT_SINGULAR


@pytest.mark.parametrize("precond", [0, 4, -1], ids=["diag", "kinetic4", "multigrid"])
@pytest.mark.parametrize("case", ["h2o_11", "h2_16"])
def test_block_davidson_vs_reference_algorithm(engine, port, case, precond):
    """Eigenpairs of the block solver vs the reference's state-by-state Davidson (oracle)."""
    if case == "h2o_11":
        n, b, Z = (11, 9, 8), (-3.0, 3.4, -2.5, 2.9, -2.2, 2.0), [8, 1, 1]
        xyz = np.array([0.05, 0.07, 0.03, 1.43, 0.07, 1.1, -1.43, 0.07, 1.1])
        nocc = 4
    else:
        # sigma_g, sigma_u (levels 3-4 are the degenerate pi_u pair: not split by nocc)
        n, b, Z = (16, 16, 16), (-6.0, 6.0) * 3, [1, 1]
        xyz = np.array([-0.7, 0.0, 0.0, 0.7, 0.0, 0.0])
        nocc = 2
    g = G(n, b)
    N = g.getSize()
    V = port.nuclear_potential(n, b, Z, xyz)
    e_ref, psi_ref = port.solve_orbitals(n, b, V, nocc)
    nbands = nocc + 3
    psi = engine.array(nbands * N)
    eig, it = engine.solve_orbitals(g, engine.upload(V), nocc, nbands, psi, N, init=False, preconditioner=precond)
    assert np.max(np.abs(eig[:nocc] - e_ref)) < 1e-9
    P = psi.to_host((nbands, N))
    dV = g.getDx() * g.getDy() * g.getDz()
    # dV-normalised, orthonormal, and the same subspace as the reference's orbitals
    S = P[:nocc] @ P[:nocc].T * dV
    assert np.max(np.abs(S - np.eye(nocc))) < 1e-10
    overlap = psi_ref @ P[:nocc].T * dV
    assert np.max(np.abs(np.abs(np.linalg.det(overlap)) - 1.0)) < 1e-6
    # KS residuals below the reference tolerance
    for k in range(nocc):
        hp = port.apply_hamiltonian(n, b, V, P[k])
        r = np.sqrt(np.sum((hp - eig[k] * P[k]) ** 2) * dV)
        assert r < 1e-7


@pytest.mark.parametrize("n", [(6, 5, 4), (48, 48, 48), (96, 96, 97)])
@pytest.mark.parametrize("ka,kb", [(1, 1), (5, 3), (20, 4), (64, 16), (33, 9)])
def test_gram_narrow_fp64(engine, n, ka, kb):
    """The one-launch narrow FP64 Gram (ka <= 64, kb <= 16; two-level in-launch reduction over
    groups of 16 blocks, the last group partial): dV * A^T B against numpy to 1e-13, and
    repeated calls are bitwise identical (fixed summation order, tickets reset)."""
    g = G(n, (-4.0, 4.0) * 3)
    N = g.getSize()
    rng = np.random.default_rng(ka * 100 + kb)
    A = rng.standard_normal((ka, N))
    B = rng.standard_normal((kb, N))
    dA, dB = engine.upload(A), engine.upload(B)
    c1 = engine.gram(g, dA, N, ka, dB, N, kb, precision=0)
    c2 = engine.gram(g, dA, N, ka, dB, N, kb, precision=0)
    dV = g.getDx() * g.getDy() * g.getDz()
    ref = (A @ B.T) * dV
    assert np.max(np.abs(np.asarray(c1) - ref)) < 1e-14 * N * dV
    assert np.array_equal(np.asarray(c1), np.asarray(c2))
