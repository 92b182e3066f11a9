"""GPU: the z-slab kernels (dft_zslab_*_dev) under the z-slab driver, all slabs held by one
process on one GPU (LocalSlabs: halos by device copies, no kernel waits on another).

The potential and sweep count of 1-4 slabs equal dft_hartree_dev / the oracle bit for bit
(HartreePotentialMolecule.cpp:99-324), from a cold and from a warm start, at the reference's
stop and at a sweep cap; H psi of 1-4 slabs equals dft_apply_hamiltonian_dev bit for bit
(KohnShamHamiltonianMolecule.cpp:78-177); the XC potentials equal dft_xc_dev bit for bit and
E_xc to 1e-12 (ExchangeCorrelationMolecule.cpp:576-842); the slabs' Gram parts add up to
dft_gram_dev's product; invalid slab arguments are rejected before any launch."""
import numpy as np
import pytest
import torch

from dft_b200 import CartesianGrid, DFTError
from dft_b200.zslab import (CudaSlabOps, LocalSlabs, SlabLayout, gram_zslab, hamiltonian_zslab, hartree_zslab,
                            xc_zslab)

pytestmark = pytest.mark.gpu

# spacing 0.25 bohr on every axis: zero boundary values
N = (33, 25, 41)
B = (-4.0, 4.0, -3.0, 3.0, -5.0, 5.0)


def _density(n, b):
    x = np.linspace(b[0], b[1], n[0])
    y = np.linspace(b[2], b[3], n[1])
    z = np.linspace(b[4], b[5], n[2])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    return (np.exp(-((X - 0.7) ** 2 + Y ** 2 + (Z + 1.1) ** 2)) +
            0.5 * np.exp(-((X + 1.0) ** 2 + (Y - 0.5) ** 2 + (Z - 2.0) ** 2) / 0.6)).ravel()


def _slab_solve(engine, n, b, rho, world, halo, max_sweeps=10000, guess=None):
    g = CartesianGrid(*n, *b)
    lay = SlabLayout(n, world, halo)
    field = torch.from_numpy(rho).cuda()
    slabs = {r: lay.scatter(field, r) for r in range(world)}
    gs = None if guess is None else {r: lay.scatter(torch.from_numpy(guess).cuda(), r) for r in range(world)}
    v, sweeps, last = hartree_zslab(LocalSlabs(world), lay, g, slabs, CudaSlabOps(engine), 1e-8, max_sweeps, gs)
    return lay.gather(v).cpu().numpy(), sweeps, last


def _whole(engine, n, b, rho, max_sweeps=10000, guess=None):
    g = CartesianGrid(*n, *b)
    d_rho = engine.upload(rho)
    if guess is None:
        d_v = engine.array(rho.size)
        sweeps, last = engine.hartree(g, d_rho, d_v, 1e-8, max_sweeps)
    else:
        d_v = engine.upload(guess)
        sweeps, last = engine.hartree_from_guess(g, d_rho, d_v, 1e-8, max_sweeps)
    return d_v.to_host(), sweeps, last


@pytest.mark.parametrize("world,halo", [(1, 8), (2, 8), (3, 5), (4, 3)])
def test_hartree_slabs_match_whole_grid(engine, port, world, halo):
    rho = _density(N, B)
    ref_v, ref_s, ref_l = _whole(engine, N, B, rho)
    v, s, l = _slab_solve(engine, N, B, rho, world, halo)
    assert s == ref_s and l == ref_l
    assert v.tobytes() == ref_v.tobytes()
    if world == 2:
        assert v.tobytes() == port.hartree_potential(N, B, rho).tobytes()


def test_hartree_slabs_warm_start_and_cap(engine):
    n, b = (96, 80, 112), (-11.875, 11.875, -9.875, 9.875, -13.875, 13.875)  # spacing 0.25
    rho = _density(n, b)
    ref_v, ref_s, _ = _whole(engine, n, b, rho, max_sweeps=200)
    v, s, _ = _slab_solve(engine, n, b, rho, 4, 8, max_sweeps=200)
    assert s == ref_s == 200
    assert v.tobytes() == ref_v.tobytes()
    guess = 0.5 * ref_v
    wv, ws, wl = _whole(engine, n, b, rho, max_sweeps=300, guess=guess)
    sv, ss, sl = _slab_solve(engine, n, b, rho, 3, 8, max_sweeps=300, guess=guess)
    assert ss == ws and sl == wl
    assert sv.tobytes() == wv.tobytes()


@pytest.mark.parametrize("world", [1, 2, 4])
def test_hamiltonian_slabs_match_whole_grid(engine, world):
    rng = np.random.default_rng(11)
    nb = 3
    npts = int(np.prod(N))
    V = rng.standard_normal(npts)
    psi = rng.standard_normal((nb, npts))
    g = CartesianGrid(*N, *B)
    dH = engine.array(nb * npts)
    engine.apply_hamiltonian(g, engine.upload(V), engine.upload(psi), dH, nb, npts)
    ref = dH.to_host((nb, npts))
    lay = SlabLayout(N, world, 1)
    Vt, Pt = torch.from_numpy(V).cuda(), torch.from_numpy(psi).cuda()
    Vs = {r: lay.scatter(Vt, r) for r in range(world)}
    Ps = {r: lay.scatter(Pt, r) for r in range(world)}
    for r in range(world):  # halo planes come from the exchange
        rows = lay.owned_rows(r)
        view = Ps[r].view(nb, -1, lay.plane_points)
        view[:, :rows.start] = float("nan")
        view[:, rows.stop:] = float("nan")
    out = lay.gather(hamiltonian_zslab(LocalSlabs(world), lay, g, Vs, Ps, nb, CudaSlabOps(engine))).cpu().numpy()
    assert out.tobytes() == ref.tobytes()


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("world", [1, 2, 4])
def test_xc_slabs_match_whole_grid(engine, kind, world):
    rho = _density(N, B)
    na, nb = 0.6 * rho, 0.4 * rho + 0.05 * np.roll(rho, 7)
    g = CartesianGrid(*N, *B)
    npts = rho.size
    dva, dvb = engine.array(npts), engine.array(npts)
    ref_e = engine.xc(g, kind, engine.upload(na), engine.upload(nb), dva, dvb)
    lay = SlabLayout(N, world, 2)
    A = {r: lay.scatter(torch.from_numpy(na).cuda(), r) for r in range(world)}
    Bs = {r: lay.scatter(torch.from_numpy(nb).cuda(), r) for r in range(world)}
    for r in range(world):  # halo planes come from the exchange
        rows = lay.owned_rows(r)
        for t in (A[r], Bs[r]):
            view = t.view(-1, lay.plane_points)
            view[:rows.start] = float("nan")
            view[rows.stop:] = float("nan")
    va, vb, exc = xc_zslab(LocalSlabs(world), lay, g, kind, A, Bs, CudaSlabOps(engine))
    assert lay.gather(va).cpu().numpy().tobytes() == dva.to_host().tobytes()
    assert lay.gather(vb).cpu().numpy().tobytes() == dvb.to_host().tobytes()
    assert abs(exc - ref_e) <= 1e-12 * abs(ref_e)


@pytest.mark.parametrize("precision", [0, 1])
def test_gram_slabs_sum_to_whole_grid(engine, precision):
    rng = np.random.default_rng(5)
    npts = int(np.prod(N))
    ka, kb = 40, 24
    A, Bm = rng.standard_normal((ka, npts)), rng.standard_normal((kb, npts))
    g = CartesianGrid(*N, *B)
    ref = engine.gram(g, engine.upload(A), npts, ka, engine.upload(Bm), npts, kb, 0)
    lay = SlabLayout(N, 3, 1)
    At, Bt = torch.from_numpy(A).cuda(), torch.from_numpy(Bm).cuda()
    As = {r: lay.scatter(At, r) for r in range(3)}
    Bs = {r: lay.scatter(Bt, r) for r in range(3)}
    c = gram_zslab(LocalSlabs(3), lay, g, As, ka, Bs, kb, CudaSlabOps(engine), precision).cpu().numpy()
    tol = 1e-12 if precision == 0 else 1e-5
    assert np.max(np.abs(c - ref)) <= tol * np.max(np.abs(ref))


def test_slab_arguments_rejected(engine):
    ops = CudaSlabOps(engine)
    g = CartesianGrid(*N, *B)
    npl = N[0] * N[1]
    t = {k: torch.zeros(10 * npl, dtype=torch.float64, device="cuda") for k in ("rho", "v", "w", "tmp")}
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(DFTError):  # owned plane 5 is the slab's first plane (no halo beyond it)
        ops.jacobi_sweeps(g, 5, 15, 5, 10, t["rho"], t["v"], t["w"], t["tmp"], 4, d)
    with pytest.raises(DFTError):  # slab past the grid
        ops.jacobi_sweeps(g, 35, 45, 36, 44, t["rho"], t["v"], t["w"], t["tmp"], 4, d)
    with pytest.raises(DFTError):  # result and scratch alias
        ops.jacobi_sweeps(g, 5, 15, 6, 14, t["rho"], t["v"], t["w"], t["w"], 4, d)
    with pytest.raises(DFTError):
        ops.hamiltonian(g, 10, 5, t["v"], t["rho"], t["tmp"], 1)
    with pytest.raises(DFTError):  # one plane beyond the owned ones: XC needs two
        ops.xc(g, 5, 15, 6, 14, 1, t["rho"], t["v"], t["w"], t["tmp"])
    with pytest.raises(DFTError):  # empty owned range
        ops.gram(g, 5, 15, 8, 8, t["v"], 1, t["w"], 1)
