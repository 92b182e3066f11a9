"""CPU: the z-slab decomposition's host logic with numpy slab arithmetic.

* partitions and layouts cover every plane once and cap the halo;
* `hartree_zslab` with 1-5 slabs held by one process gives the oracle's potential and sweep
  count bit for bit (oracle_hartree_potential_ex, HartreePotentialMolecule.cpp:99-324), for
  halo widths that put the stop inside a block and at its end, and at the sweep cap;
* `hamiltonian_zslab` gives the oracle's H psi bit for bit (hpsi3,
  KohnShamHamiltonianMolecule.cpp:78-177);
* `xc_zslab` gives the oracle's XC potentials of both spins and E_xc (to rounding: the oracle
  runs on the slab as its own grid), `gram_zslab` the whole grid's Gram product;
* two and three gloo ranks (ProcessGroupSlabs: batched point-to-point halos, MAX and SUM
  all-reduces) give the same results as one process."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from dft_b200 import CartesianGrid
from dft_b200.zslab import (LocalSlabs, SlabLayout, gram_zslab, hamiltonian_zslab, hartree_zslab, owned_planes,
                            xc_zslab)

from tests.zslab_numpy import NumpySlabOps

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# spacings of 0.5 bohr: every face's last node lands on its bound (zero boundary values)
N = (17, 13, 21)
B = (-4.0, 4.0, -3.0, 3.0, -5.0, 5.0)


def _density(n=N, b=B):
    x = np.linspace(b[0], b[1], n[0])
    y = np.linspace(b[2], b[3], n[1])
    z = np.linspace(b[4], b[5], n[2])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rho = np.exp(-((X - 0.7) ** 2 + Y ** 2 + (Z + 1.1) ** 2)) + 0.5 * np.exp(-((X + 1.0) ** 2 + (Y - 0.5) ** 2 + (Z - 2.0) ** 2) / 0.6)
    return rho.ravel()


def _oracle_hartree(port, n, b, rho):
    out = np.empty_like(rho)
    sw = C.c_long()
    ld = C.c_double()
    port.check(port.fn("hartree_potential_ex")(np.asarray(n, dtype=np.int64).ctypes.data_as(C.POINTER(C.c_long)),
                                               np.asarray(b, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                               rho.ctypes.data_as(C.POINTER(C.c_double)),
                                               out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(sw), C.byref(ld)))
    return out, sw.value, ld.value


def _solve_local(world, halo, rho, tol=1e-8, max_sweeps=10000, n=N, b=B):
    g = CartesianGrid(*n, *b)
    lay = SlabLayout(n, world, halo)
    field = torch.from_numpy(rho)
    slabs = {r: lay.scatter(field, r) for r in range(world)}
    v, sweeps, last = hartree_zslab(LocalSlabs(world), lay, g, slabs, NumpySlabOps(), tol, max_sweeps)
    return lay.gather(v).numpy(), sweeps, last


def test_owned_planes_cover_once():
    for nz in (2, 3, 7, 64, 193):
        for world in range(1, min(nz, 9) + 1):
            runs = owned_planes(nz, world)
            assert runs[0][0] == 0 and runs[-1][1] == nz
            assert all(runs[r][1] == runs[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in runs]
            assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        owned_planes(3, 4)


def test_layout_halo_capped_by_smallest_run():
    lay = SlabLayout((8, 8, 10), 4, 8)  # runs of 3, 3, 2, 2 planes
    assert lay.halo == 2
    assert lay.extent(0) == (0, 5) and lay.extent(3) == (6, 10)
    assert lay.owned_rows(1) == slice(2, 5)


def test_exchange_wider_than_halo_rejected():
    lay = SlabLayout(N, 3, 1)
    t = {r: torch.zeros(lay.points(r), dtype=torch.float64) for r in range(3)}
    with pytest.raises(ValueError):
        LocalSlabs(3).exchange(lay, t, 2)


def test_hartree_single_slab_is_the_oracle(port):
    rho = _density()
    ref, sw, ld = _oracle_hartree(port, N, B, rho)
    v, sweeps, last = _solve_local(1, 8, rho)
    assert sweeps == sw and last == ld
    assert v.tobytes() == ref.tobytes()


@pytest.mark.parametrize("world,halo", [(2, 8), (3, 5), (4, 1), (5, 3), (3, 64)])
def test_hartree_slabs_bit_identical(port, world, halo):
    rho = _density()
    ref, sw, ld = _oracle_hartree(port, N, B, rho)
    v, sweeps, last = _solve_local(world, halo, rho)
    assert sweeps == sw and last == ld
    assert v.tobytes() == ref.tobytes()


def test_hartree_cap_and_zero_sweeps():
    rho = _density()
    one, s1, l1 = _solve_local(1, 7, rho, max_sweeps=37)
    three, s3, l3 = _solve_local(3, 7, rho, max_sweeps=37)
    assert s1 == s3 == 37 and l1 == l3
    assert three.tobytes() == one.tobytes()
    z, s0, _ = _solve_local(3, 4, rho, max_sweeps=0)
    assert s0 == 0 and not z.any()


def test_hartree_one_plane_per_rank(port):
    # nz ranks: halo 1, an exchange every sweep; the first and last rank own only a face
    n, b = (9, 8, 6), (-2.0, 2.0, -1.75, 1.75, -1.25, 1.25)
    rho = _density(n, b)
    ref, sw, ld = _oracle_hartree(port, n, b, rho)
    v, sweeps, last = _solve_local(6, 4, rho, n=n, b=b)
    assert sweeps == sw and last == ld
    assert v.tobytes() == ref.tobytes()


def test_hartree_warm_start():
    rho = _density()
    g = CartesianGrid(*N, *B)
    start, _, _ = _solve_local(1, 8, rho, max_sweeps=50)
    guess = torch.from_numpy(0.9 * start)
    out = {}
    for world in (1, 3):
        lay = SlabLayout(N, world, 6)
        slabs = {r: lay.scatter(torch.from_numpy(rho), r) for r in range(world)}
        gs = {r: lay.scatter(guess, r) for r in range(world)}
        v, sweeps, last = hartree_zslab(LocalSlabs(world), lay, g, slabs, NumpySlabOps(), 1e-8, 10000, gs)
        out[world] = (lay.gather(v).numpy().tobytes(), sweeps, last)
    assert out[1] == out[3]


def test_hartree_faces_off_the_nodes_close():
    # 0.6/7 spacing misses the bound by rounding: Q/|r| face values, Q summed per rank
    n, b = (8, 9, 15), (-3.0, 3.3, -3.1, 3.0, -4.0, 4.2)
    rho = _density(n, b)
    one, s1, _ = _solve_local(1, 4, rho, n=n, b=b)
    three, s3, _ = _solve_local(3, 4, rho, n=n, b=b)
    assert abs(s1 - s3) <= 1
    assert np.max(np.abs(three - one)) <= 1e-12 * np.max(np.abs(one))


@pytest.mark.parametrize("world", [1, 2, 4])
def test_hamiltonian_slabs_bit_identical(port, world):
    rng = np.random.default_rng(7)
    nb = 3
    V = rng.standard_normal(int(np.prod(N)))
    psi = rng.standard_normal((nb, int(np.prod(N))))
    g = CartesianGrid(*N, *B)
    lay = SlabLayout(N, world, 1)
    Vs = {r: lay.scatter(torch.from_numpy(V), r) for r in range(world)}
    Ps = {r: lay.scatter(torch.from_numpy(psi), r) for r in range(world)}
    for r in range(world):  # halo planes come from the exchange, not from the scatter
        rows = lay.owned_rows(r)
        view = Ps[r].view(nb, -1, lay.plane_points)
        view[:, :rows.start] = np.nan
        view[:, rows.stop:] = np.nan
    out = lay.gather(hamiltonian_zslab(LocalSlabs(world), lay, g, Vs, Ps, nb, NumpySlabOps())).numpy()
    for k in range(nb):
        assert out[k].tobytes() == port.apply_hamiltonian(N, B, V, psi[k]).tobytes(), k


def _spin_densities(n=N, b=B):
    rho = _density(n, b)
    x = np.linspace(b[0], b[1], n[0])
    Z, Y, X = np.meshgrid(np.linspace(b[4], b[5], n[2]), np.linspace(b[2], b[3], n[1]), x, indexing="ij")
    return 0.6 * rho, 0.4 * rho + 0.05 * np.exp(-((X - 1.5) ** 2 + Y ** 2 + Z ** 2)).ravel()


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("world", [1, 2, 3])
def test_xc_slabs_match_oracle(port, kind, world):
    na, nb = _spin_densities()
    g = CartesianGrid(*N, *B)
    lay = SlabLayout(N, world, 2)
    A = {r: lay.scatter(torch.from_numpy(na), r) for r in range(world)}
    Bs = {r: lay.scatter(torch.from_numpy(nb), r) for r in range(world)}
    va, vb, exc = xc_zslab(LocalSlabs(world), lay, g, kind, A, Bs, NumpySlabOps(port))
    for v, spin in ((lay.gather(va).numpy(), 0), (lay.gather(vb).numpy(), 1)):
        ref = port.xc_potential(kind, N, B, na, nb, spin)
        assert np.max(np.abs(v - ref)) <= 1e-12 * np.max(np.abs(ref)), spin
    ref_e = port.xc_energy(kind, N, B, na, nb)
    assert abs(exc - ref_e) <= 1e-12 * abs(ref_e)


def test_xc_needs_two_halo_planes():
    g = CartesianGrid(*N, *B)
    lay = SlabLayout(N, 3, 1)
    t = {r: torch.zeros(lay.points(r), dtype=torch.float64) for r in range(3)}
    with pytest.raises(ValueError):
        xc_zslab(LocalSlabs(3), lay, g, 1, t, dict(t), NumpySlabOps())


@pytest.mark.parametrize("world", [1, 2, 4])
def test_gram_slabs_sum_to_whole_grid(world):
    rng = np.random.default_rng(3)
    npts = int(np.prod(N))
    A, Bm = rng.standard_normal((5, npts)), rng.standard_normal((3, npts))
    g = CartesianGrid(*N, *B)
    lay = SlabLayout(N, world, 1)
    As = {r: lay.scatter(torch.from_numpy(A), r) for r in range(world)}
    Bs = {r: lay.scatter(torch.from_numpy(Bm), r) for r in range(world)}
    for r in range(world):  # halo planes are not read
        rows = lay.owned_rows(r)
        for t in (As[r], Bs[r]):
            view = t.view(t.shape[0], -1, lay.plane_points)
            view[:, :rows.start] = np.nan
            view[:, rows.stop:] = np.nan
    c = gram_zslab(LocalSlabs(world), lay, g, As, 5, Bs, 3, NumpySlabOps()).numpy()
    ref = (A @ Bm.T) * (g.getDx() * g.getDy() * g.getDz())
    assert np.max(np.abs(c - ref)) <= 1e-12 * np.max(np.abs(ref))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port_no, out_dir):
    import sys

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from tests.zslab_numpy import NumpySlabOps as Ops
    from dft_b200.zslab import ProcessGroupSlabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port_no))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        comm = ProcessGroupSlabs()
        g = CartesianGrid(*N, *B)
        lay = SlabLayout(N, world, 5)
        rho = torch.from_numpy(_density())
        v, sweeps, last = hartree_zslab(comm, lay, g, {rank: lay.scatter(rho, rank)}, Ops())
        rows = lay.owned_rows(rank)
        n = lay.plane_points
        np.save(os.path.join(out_dir, f"v{rank}.npy"), v[rank][rows.start * n:rows.stop * n].numpy())
        rng = np.random.default_rng(7)
        V = torch.from_numpy(rng.standard_normal(int(np.prod(N))))
        psi = torch.from_numpy(rng.standard_normal((2, int(np.prod(N)))))
        lay1 = SlabLayout(N, world, 1)
        h = hamiltonian_zslab(comm, lay1, g, {rank: lay1.scatter(V, rank)}, {rank: lay1.scatter(psi, rank)}, 2, Ops())
        rows = lay1.owned_rows(rank)
        np.save(os.path.join(out_dir, f"h{rank}.npy"), h[rank][:, rows.start * n:rows.stop * n].numpy())
        na, nb = (torch.from_numpy(x) for x in _spin_densities())
        lay2 = SlabLayout(N, world, 2)
        va, vb, exc = xc_zslab(comm, lay2, g, 1, {rank: lay2.scatter(na, rank)}, {rank: lay2.scatter(nb, rank)}, Ops())
        rows = lay2.owned_rows(rank)
        np.save(os.path.join(out_dir, f"x{rank}.npy"), va[rank][rows.start * n:rows.stop * n].numpy())
        c = gram_zslab(comm, lay1, g, {rank: lay1.scatter(psi, rank)}, 2, {rank: lay1.scatter(psi, rank)}, 2, Ops())
        np.save(os.path.join(out_dir, f"c{rank}.npy"), c.numpy())
        with open(os.path.join(out_dir, f"s{rank}.txt"), "w") as f:
            f.write(f"{sweeps} {last!r} {exc!r}")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks(port, tmp_path, world):
    # with three ranks the middle one exchanges with both neighbours in one batch
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    rho = _density()
    ref, sw, ld = _oracle_hartree(port, N, B, rho)
    v = np.concatenate([np.load(tmp_path / f"v{r}.npy") for r in range(world)])
    assert v.tobytes() == ref.tobytes()
    na, nb = _spin_densities()
    ref_e = port.xc_energy(1, N, B, na, nb)
    excs = []
    for r in range(world):
        s, last, exc = open(tmp_path / f"s{r}.txt").read().split()
        assert int(s) == sw and float(last) == ld
        excs.append(float(exc))
    assert len(set(excs)) == 1 and abs(excs[0] - ref_e) <= 1e-12 * abs(ref_e)
    va = np.concatenate([np.load(tmp_path / f"x{r}.npy") for r in range(world)])
    ref_v = port.xc_potential(1, N, B, na, nb, 0)
    assert np.max(np.abs(va - ref_v)) <= 1e-12 * np.max(np.abs(ref_v))
    rng = np.random.default_rng(7)
    V = rng.standard_normal(int(np.prod(N)))
    psi = rng.standard_normal((2, int(np.prod(N))))
    h = np.concatenate([np.load(tmp_path / f"h{r}.npy") for r in range(world)], axis=1)
    for k in range(2):
        assert h[k].tobytes() == port.apply_hamiltonian(N, B, V, psi[k]).tobytes()
    cs = [np.load(tmp_path / f"c{r}.npy") for r in range(world)]
    g = CartesianGrid(*N, *B)
    ref_c = (psi @ psi.T) * (g.getDx() * g.getDy() * g.getDz())
    assert all(c.tobytes() == cs[0].tobytes() for c in cs)
    assert np.max(np.abs(cs[0] - ref_c)) <= 1e-12 * np.max(np.abs(ref_c))


def _rank_leaves(rank, world, port_no, out_dir):
    import datetime
    import sys
    import time

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from tests.zslab_numpy import NumpySlabOps as Ops
    from dft_b200.zslab import ProcessGroupSlabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port_no))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        return  # leaves between steps, before the solve's first exchange
    t0 = time.time()
    try:
        g = CartesianGrid(*N, *B)
        lay = SlabLayout(N, world, 4)
        hartree_zslab(ProcessGroupSlabs(), lay, g, {0: lay.scatter(torch.from_numpy(_density()), 0)}, Ops())
        outcome = "finished"
    except Exception as e:  # the exchange or the reduction with the missing rank fails
        outcome = "error " + type(e).__name__
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write(f"{outcome} {time.time() - t0:.1f}")


def test_gloo_rank_leaving_ends_the_solve_with_an_error(tmp_path):
    mp.start_processes(_rank_leaves, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    outcome, seconds = open(tmp_path / "rank0.txt").read().rsplit(" ", 1)
    assert outcome.startswith("error"), outcome
    assert float(seconds) < 60.0
