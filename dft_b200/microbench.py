"""Per-operator timings of libdft_b200 on one GPU (CUDA events on the library's stream).

    python -m dft_b200.microbench hpsi   --n 192 --bands 16 [--reps 5]
    python -m dft_b200.microbench jacobi --n 48  [--sweeps 10000]
    python -m dft_b200.microbench xc     --n 128 --functional PBE96
    python -m dft_b200.microbench scf    --n 48  [--iterations 1]     # H2 at h = 0.3 (n = 48)
    python -m dft_b200.microbench radial                              # 60 atoms, one launch
    python -m dft_b200.microbench gram   --n 64 --ka 64 --kb 64 --precision 1   # tcgen05 Gram
    python -m dft_b200.microbench poisson --n 128 --poisson multigrid [--train 32]
    python -m dft_b200.microbench train --n 96 --tc 1                 # network training step
    python -m dft_b200.microbench rotate --n 64 --ka 128 --kb 64 --precision 1   # tcgen05 rotation
    python -m dft_b200.microbench scf --system h2o_128 --poisson multigrid --mixed 1 --stop-abs-de 1e-6
    python -m dft_b200.microbench zslab --n 192 --sweeps 2000 --slabs 1,2,4 --halo 8   # z-slab Jacobi, one GPU

Each mode prints one JSON line with the time and the achieved bandwidth for the
operator's algorithmic bytes.  Used for roofline numbers and as the command under ncu.
"""
from __future__ import annotations

import argparse
import json
import statistics

import numpy as np

import dft_b200 as d


def _events(torch, stream, fn, reps, flush=None):
    times = []
    for _ in range(reps):
        with torch.cuda.stream(stream):
            if flush is not None:
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        fn()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return times


POISSON = {"cold": 0, "previous": 1, "network": 2, "coarse": 3, "hybrid": 4, "multigrid": 5}


def train_net(eng, grid, samples):
    """A network trained on the device on synthetic densities on `grid` (untimed setup)."""
    net = d.PoissonNet(eng, seed=7)
    rep = net.train([grid], samples=samples, validation=max(2, samples // 8), epochs=10, batch=4, lr=3e-3,
                    lr_min=1e-4, seed=2027, smooth_sweeps=0, mse_weight=1.0)
    return net, rep


def cube(n, h):
    half = 0.5 * h * (n - 1)
    return d.CartesianGrid(n, n, n, -half, half, -half, half, -half, half)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["hpsi", "jacobi", "xc", "scf", "radial", "gram", "poisson", "train", "rotate",
                                     "c4", "zslab"])
    ap.add_argument("--samples", type=int, default=512, help="c4: training densities")
    ap.add_argument("--held-out", type=int, default=6, help="c4: held-out densities per grid")
    ap.add_argument("--tc", type=int, default=1, help="network convolutions on the tensor cores (1) or CUDA cores (0)")
    ap.add_argument("--ka", type=int, default=64)
    ap.add_argument("--kb", type=int, default=64)
    ap.add_argument("--precision", type=int, default=0, help="gram: 0 = FP64, 1 = tensor cores (TF32 hi+lo)")
    ap.add_argument("--mixed", type=int, default=0, help="scf: mixed-precision eigensolver")
    ap.add_argument("--poisson", default="cold", choices=sorted(POISSON),
                    help="scf/poisson: start of each Poisson solve")
    ap.add_argument("--precond", type=int, default=4,
                    help="scf: eigensolver preconditioner (0 diagonal, k > 0 smoothing steps, -1 multigrid)")
    ap.add_argument("--mixer", type=int, default=0, help="scf: 0 linear (reference), 1 Pulay")
    ap.add_argument("--adaptive", type=int, default=0, help="scf: adaptive eigensolver tolerance")
    ap.add_argument("--smearing", type=float, default=0.0, help="scf: Fermi-Dirac temperature (Ha), 0 = aufbau")
    ap.add_argument("--train", type=int, default=0,
                    help="scf/poisson with a network start: train on this many synthetic densities first")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--h", type=float, default=0.2)
    ap.add_argument("--bands", type=int, default=16)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--sweeps", type=int, default=10000)
    ap.add_argument("--iterations", type=int, default=1)
    ap.add_argument("--functional", default="PBE96")
    ap.add_argument("--spl", type=int, default=0, help="Jacobi sweeps per launch (0 = auto)")
    ap.add_argument("--bpt", type=int, default=0, help="H psi bands per thread (0 = auto)")
    ap.add_argument("--ring", type=int, default=0, help="tensor-core Gram through the cp.async ring (1)")
    ap.add_argument("--system", default="h2_48", help="scf mode: h2_48, h2o_128, cluster20")
    ap.add_argument("--stop-abs-de", type=float, default=0.0)
    ap.add_argument("--stop-abs-deig", type=float, default=0.0)
    ap.add_argument("--kerker", type=float, default=0.0, help="scf: Kerker screening q0 (bohr^-1), 0 = off")
    ap.add_argument("--atoms", type=int, default=0, help="scf: superposed-atoms start (1)")
    ap.add_argument("--pulay-beta", type=float, default=0.0, help="scf: Pulay step (0 = 0.5)")
    ap.add_argument("--pulay-depth", type=int, default=0, help="scf: Pulay history (0 = 16)")
    ap.add_argument("--boundary", type=int, default=0, help="scf: Hartree faces, 0 reference, 1 Q/|r| (monopole)")
    ap.add_argument("--predict", type=int, default=0, help="scf: V_H(n_in) start from the mixer's combination (1)")
    ap.add_argument("--tuning", default="", help="context tuning keys, e.g. orthonormalise_adaptive=0,hpsi_variant=2")
    ap.add_argument("--system-args", default="{}", help='scf: JSON keyword arguments of the system, e.g. {"nmol": 7}')
    ap.add_argument("--slabs", default="1,2,4", help="zslab: slab counts (all slabs held by this process)")
    ap.add_argument("--halo", type=int, default=8, help="zslab: halo planes per side (sweeps per exchange)")
    ap.add_argument("--verbose", type=int, default=0)
    a = ap.parse_args()
    import torch

    eng = d.Engine(0)
    for kv in filter(None, a.tuning.split(",")):
        key, val = kv.split("=")
        eng.set_tuning(key.strip(), int(val))
    eng.set_tuning("jacobi_sweeps_per_launch", a.spl)
    eng.set_tuning("network_tensor_cores", a.tc)
    eng.set_tuning("hpsi_bands_per_thread", a.bpt)
    eng.set_tuning("tensor_core_ring", a.ring)
    stream = torch.cuda.ExternalStream(eng.stream)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {"mode": a.mode}
    if a.mode == "hpsi":
        g = cube(a.n, a.h)
        N = g.getSize()
        V, P, H = eng.array(N), eng.array(N * a.bands), eng.array(N * a.bands)
        t = _events(torch, stream, lambda: eng.apply_hamiltonian(g, V, P, H, a.bands, N), a.reps, flush)
        ms = statistics.median(t)
        byts = (16.0 + 8.0 / a.bands) * N * a.bands
        out.update(n=a.n, bands=a.bands, ms=ms, gbs=byts / (ms * 1e-3) / 1e9, bytes=byts)
    elif a.mode == "jacobi":
        g = cube(a.n, a.h)
        N = g.getSize()
        x = np.linspace(-1, 1, a.n)
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        rho = eng.upload(np.exp(-8 * (X ** 2 + Y ** 2 + Z ** 2)).ravel())
        vh = eng.array(N)
        res = {}

        def run():
            res["s"] = eng.hartree(g, rho, vh, 1e-8, a.sweeps)[0]

        t = _events(torch, stream, run, a.reps)
        ms = statistics.median(t)
        interior = (a.n - 2) ** 3
        out.update(n=a.n, spl=a.spl, sweeps=res["s"], ms=ms, us_per_sweep=1e3 * ms / res["s"],
                   gbs=24.0 * interior * res["s"] / (ms * 1e-3) / 1e9)
    elif a.mode == "zslab":
        # wall time: the slab driver is host-synchronous (one exchange and one reduction per block)
        import time

        from .zslab import CudaSlabOps, LocalSlabs, SlabLayout, hartree_zslab
        g = cube(a.n, a.h)
        N = g.getSize()
        x = np.linspace(-1, 1, a.n)
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        rho_h = np.exp(-8 * (X ** 2 + Y ** 2 + Z ** 2)).ravel()
        rho, vh = eng.upload(rho_h), eng.array(N)
        eng.hartree(g, rho, vh, 1e-8, min(a.sweeps, 64))
        t0 = time.perf_counter()
        s_ref, _ = eng.hartree(g, rho, vh, 1e-8, a.sweeps)
        whole_ms = 1e3 * (time.perf_counter() - t0)
        ref = vh.to_host()
        field = torch.from_numpy(rho_h).cuda()
        ops = CudaSlabOps(eng)
        rows = []
        for R in [int(v) for v in a.slabs.split(",")]:
            lay = SlabLayout(g.shape, R, a.halo)
            sl = {r: lay.scatter(field, r) for r in range(R)}
            hartree_zslab(LocalSlabs(R), lay, g, sl, ops, 1e-8, min(a.sweeps, 4 * lay.halo))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            v, s, _ = hartree_zslab(LocalSlabs(R), lay, g, sl, ops, 1e-8, a.sweeps)
            torch.cuda.synchronize()
            ms = 1e3 * (time.perf_counter() - t0)
            same = bool(s == s_ref and lay.gather(v).cpu().numpy().tobytes() == ref.tobytes())
            rows.append({"slabs": R, "halo": lay.halo, "sweeps": s, "ms": ms, "us_per_sweep": 1e3 * ms / s,
                         "identical_to_whole_grid": same})
            del v, sl
        out.update(n=a.n, sweeps=s_ref, whole_ms=whole_ms, whole_us_per_sweep=1e3 * whole_ms / s_ref, slabs=rows)
    elif a.mode == "xc":
        g = cube(a.n, a.h)
        N = g.getSize()
        x = np.linspace(-1, 1, a.n)
        X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
        r2 = (X ** 2 + Y ** 2 + Z ** 2).ravel()
        na, nb = eng.upload(np.exp(-6 * r2)), eng.upload(0.7 * np.exp(-5 * r2))
        va, vb = eng.array(N), eng.array(N)
        t = _events(torch, stream, lambda: eng.xc(g, a.functional, na, nb, va, vb, energy=True), a.reps, flush)
        ms = statistics.median(t)
        out.update(n=a.n, functional=a.functional, ms=ms, gpoints_per_s=N / (ms * 1e-3) / 1e9,
                   gbs=32.0 * N / (ms * 1e-3) / 1e9)
    elif a.mode == "scf":
        from dft_b200 import systems
        w = systems.get(a.system, **json.loads(a.system_args))
        g = d.CartesianGrid(*w["n"], *w["bounds"])
        m = d.Molecule()
        for z, p in zip(w["Z"], w["xyz"]):
            m.addNucleus(z, *p)
        net, rep = (None, None)
        if a.train:
            net, rep = train_net(eng, g, a.train)
            out["train"] = {k: rep[k] for k in ("steps", "seconds_data", "seconds_train", "val_loss",
                                                "val_loss_coarse")}
        o = d.default_scf_options(max_iterations=a.iterations, extra_bands=w["extra_bands"], verbose=int(a.verbose),
                                  stop_abs_de=a.stop_abs_de, stop_abs_deig=a.stop_abs_deig,
                                  poisson_start=POISSON[a.poisson], mixer=a.mixer, adaptive_eig_tol=a.adaptive,
                                  smearing_kt=a.smearing, kerker_q0=a.kerker, initial_density=a.atoms,
                                  pulay_beta=a.pulay_beta, pulay_depth=a.pulay_depth,
                                  hartree_boundary=a.boundary, poisson_predict=a.predict)
        if net is not None:
            o.poisson_net = net.handle
        o.eig.verbose = int(a.verbose > 2)
        o.eig.mixed_precision = a.mixed
        o.eig.preconditioner = a.precond
        r = eng.scf_molecule(g, m, 0, w["multiplicity"], w["functional"], o)
        out.update(system=a.system, poisson=a.poisson, mixed=a.mixed, precond=a.precond, iterations=r.iterations,
                   converged=r.converged,
                   energy=r.total,
                   seconds=r.seconds, launches=eng.launches,
                   tensor_core_products=eng.counter("tensor_core_products"), eigenvalues=r.eigenvalues[:8],
                   history=[{k: h[k] for k in ("iteration", "energy", "energy_difference", "density_difference",
                                               "ks_residual", "eigenvalue_difference", "poisson_sweeps_in",
                                               "poisson_sweeps_out", "poisson_cycles_in", "poisson_cycles_out",
                                               "eig_iterations_alpha", "ms_hartree", "ms_xc", "ms_orbitals",
                                               "ms_density", "ms_energy", "ms_total")} for h in r.history])
    elif a.mode == "poisson":
        g = cube(a.n, a.h)
        N = g.getSize()
        rho, v = eng.array(N), eng.array(N)
        eng.synthetic_density(g, 5, rho)
        net = train_net(eng, g, a.train)[0] if a.train else None
        res = {}

        def run():
            if a.poisson == "cold":
                res["s"] = eng.hartree(g, rho, v)[0]
                res["c"] = 0
            else:
                cyc = 40 if a.poisson == "multigrid" else 0
                info = eng.poisson_start(g, net, rho, v, multigrid_cycles=cyc)
                res["c"] = info["multigrid_cycles"] + info["coarse_cycles"]
                res["s"] = eng.hartree_from_guess(g, rho, v)[0]

        t = _events(torch, stream, run, a.reps)
        out.update(n=a.n, poisson=a.poisson, network=bool(net), ms=statistics.median(t), sweeps=res["s"],
                   cycles=res["c"])
    elif a.mode == "c4":
        # the learned Poisson start at the scale of the learned-start workload: seeded synthetic
        # densities (1-8 Gaussians, widths 0.3-2 bohr, 2-40 electrons) on 96^3 and 128^3 grids at
        # h = 0.2, targets the Jacobi fixed point to 1e-10; then, on held-out densities, the
        # Jacobi sweeps (reference stop rule: max|dV| < 1e-8, cap 10000) and the final max error
        # against the fixed point from each start
        import time
        grids = [cube(96, a.h), cube(128, a.h)]
        net = d.PoissonNet(eng, seed=7)
        t0 = time.perf_counter()
        rep = net.train(grids, samples=a.samples, validation=max(8, a.samples // 16), epochs=10, batch=4, lr=3e-3,
                        lr_min=1e-4, seed=2029, smooth_sweeps=0, mse_weight=1.0)
        train_s = time.perf_counter() - t0
        starts = {}
        for g in grids:
            N = g.getSize()
            rho, v, vstar = eng.array(N), eng.array(N), eng.array(N)
            for q in range(a.held_out):
                eng.synthetic_density(g, 900000 + 17 * q + g.nx, rho)
                eng.poisson_start(g, None, rho, vstar, multigrid_cycles=60)
                eng.hartree_from_guess(g, rho, vstar, 1e-10, 400000)
                ref = vstar.to_host()
                for name in ("cold", "coarse", "coarse+network", "multigrid+network"):
                    if name == "cold":
                        sw = eng.hartree(g, rho, v, 1e-8, 10000)[0]
                    else:
                        eng.poisson_start(g, net if "network" in name else None, rho, v,
                                          multigrid_cycles=40 if name.startswith("multigrid") else 0)
                        sw = eng.hartree_from_guess(g, rho, v, 1e-8, 10000)[0]
                    err = float(np.max(np.abs(v.to_host() - ref)))
                    st = starts.setdefault(f"{g.nx}^3 {name}", {"sweeps": [], "max_error": []})
                    st["sweeps"].append(sw)
                    st["max_error"].append(err)
        summary = {k: {"mean_sweeps": float(np.mean(v["sweeps"])), "mean_max_error": float(np.mean(v["max_error"])),
                       "capped": int(sum(1 for x in v["sweeps"] if x >= 10000))} for k, v in starts.items()}
        out.update(samples=a.samples, grids=[96, 128], h=a.h, train_seconds=train_s, steps=rep["steps"],
                   val_loss=rep["val_loss"], val_loss_coarse=rep["val_loss_coarse"],
                   mean_target_sweeps=rep["mean_target_sweeps"], held_out_per_grid=a.held_out, starts=summary)
    elif a.mode == "rotate":
        g = cube(a.n, a.h)
        N = g.getSize()
        k, m = a.ka, a.kb
        rng = np.random.default_rng(0)
        V = eng.upload(rng.standard_normal(N * k))
        X = eng.array(N * m)
        Y = rng.standard_normal((k, m))
        t = _events(torch, stream, lambda: eng.rotate(g, V, N, k, Y, X, N, precision=a.precision), a.reps, flush)
        ms = statistics.median(t)
        out.update(n=a.n, k=k, m=m, precision=a.precision, ms=ms, tflops=2.0 * N * k * m / (ms * 1e-3) / 1e12,
                   gbs=8.0 * N * (k + m) / (ms * 1e-3) / 1e9)
    elif a.mode == "train":
        g = cube(a.n, a.h)
        net = d.PoissonNet(eng, seed=7)
        rep = net.train([g], samples=16, validation=4, epochs=3, batch=4, lr=3e-3, lr_min=1e-4, seed=5,
                        smooth_sweeps=0, mse_weight=1.0)
        out.update(n=a.n, tc=a.tc, ms_per_step=rep["ms_per_step"], samples_per_step=4, steps=rep["steps"],
                   seconds_data=rep["seconds_data"], val_loss=rep["val_loss"], val_loss_coarse=rep["val_loss_coarse"])
    elif a.mode == "gram":
        g = cube(a.n, a.h)
        N = g.getSize()
        ka, kb = a.ka, a.kb
        rng = np.random.default_rng(0)
        A = eng.upload(rng.standard_normal(N * ka))
        B = eng.upload(rng.standard_normal(N * kb))
        t = _events(torch, stream, lambda: eng.gram(g, A, N, ka, B, N, kb, precision=a.precision), a.reps, flush)
        ms = statistics.median(t)
        flops = 2.0 * N * ka * kb
        out.update(n=a.n, ka=ka, kb=kb, precision=a.precision, ms=ms, tflops=flops / (ms * 1e-3) / 1e12,
                   gbs=8.0 * N * (ka + kb) / (ms * 1e-3) / 1e9)
    elif a.mode == "radial":
        Zs = list(range(1, 31)) * 2
        ks = ["PZ81"] * 30 + ["PBE96"] * 30
        res = {}

        def run():
            res["r"] = eng.solve_atoms(Zs, ks)

        t = _events(torch, stream, run, max(1, a.reps // 2))
        ms = statistics.median(t)
        out.update(runs=60, ms=ms, runs_per_s=60 / (ms * 1e-3),
                   max_iterations=max(r.iterations for r in res["r"]))
    print(json.dumps(out), flush=True)
    eng.close()


if __name__ == "__main__":
    main()
