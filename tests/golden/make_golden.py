"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference sources compiled by oracle/Makefile (oracle/_ref/libdft_ref.so,
built from a checkout of willandru/DFT) and writes small JSON fixtures that the GPU
tests read on machines where the reference tree is absent.

    python tests/golden/make_golden.py radial        # 60 atoms, ~30 s
    python tests/golden/make_golden.py scf_small     # small molecular SCFs, ~1 min
    python tests/golden/make_golden.py scf_h2_48     # H2 on 48^3 (h=0.3), ~12 min
    python tests/golden/make_golden.py ops           # operator fixtures on small grids

Inputs for the operator fixtures are seeded (numpy default_rng) so they can be
rebuilt bit-for-bit.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.bindings import PBE96, PZ81, Ref  # noqa: E402

SYMBOLS = ["", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl",
           "Ar", "K", "Ca", "Sc", "Ti", "V", "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn"]

# Molecular cases: name -> (n, bounds, Z, xyz, charge, multiplicity, functional)
SCF_SMALL = {
    # the reference demo driver's H2 and H2O/N2/O2 cases (main.cpp:74-117, :124-174, :238-331)
    "h2_7_pz81": ((7, 7, 7), (-8.1, 7.9) * 3, [1, 1], [[-0.7, 0, 0], [0.7, 0, 0]], 0, 1, PZ81),
    "h2o_9_pz81": ((9, 9, 9), (-8.1, 7.9) * 3, [8, 1, 1], [[0, 0, 0], [1.430, 0, 1.108], [-1.430, 0, 1.108]],
                   0, 1, PZ81),
    "n2_9_pz81": ((9, 9, 9), (-8.1, 7.9) * 3, [7, 7], [[-1.037, 0, 0], [1.037, 0, 0]], 0, 1, PZ81),
    "o2_9_pz81_triplet": ((9, 9, 9), (-8.1, 7.9) * 3, [8, 8], [[-1.14, 0, 0], [1.14, 0, 0]], 0, 3, PZ81),
    # H2 at the 48^3 geometry on coarser centred grids, both functionals
    "h2_16_pz81": ((16, 16, 16), (-6.0, 6.0) * 3, [1, 1], [[-0.7, 0, 0], [0.7, 0, 0]], 0, 1, PZ81),
    "h2_16_pbe96": ((16, 16, 16), (-6.0, 6.0) * 3, [1, 1], [[-0.7, 0, 0], [0.7, 0, 0]], 0, 1, PBE96),
    # an open-shell chain: 3 electrons, multiplicity 2 (2 alpha + 1 beta)
    "h3_14_pbe96_doublet": ((14, 13, 12), (-5.2, 5.2, -4.8, 4.8, -4.4, 4.4), [1, 1, 1],
                            [[-1.6, 0.05, 0.02], [0.0, 0.05, 0.02], [1.6, 0.05, 0.02]], 0, 2, PBE96),
}

SCF_C1 = {
    # H2, two Z=1 nuclei at +-0.7 bohr on x, 48^3 grid with h = 0.3 on a centred box, PZ81, multiplicity 1
    "h2_48_pz81": ((48, 48, 48), (-7.05, 7.05) * 3, [1, 1], [[-0.7, 0, 0], [0.7, 0, 0]], 0, 1, PZ81),
}


def dump(name, obj):
    path = os.path.join(HERE, name)
    with open(path, "w") as f:
        json.dump(obj, f, indent=1)
    print("wrote", path)


def radial():
    ref = Ref()
    out = {"points": 2000, "rmax": 30.0, "runs": []}
    for kind, fname in ((PZ81, "PZ81"), (PBE96, "PBE96")):
        for Z in range(1, 31):
            t = time.time()
            r = ref.solve_atom(Z, kind)
            r.update({"Z": Z, "symbol": SYMBOLS[Z], "functional": fname, "seconds": time.time() - t,
                      "configuration": ref.atomic_configuration(Z)})
            out["runs"].append(r)
            print(fname, Z, r["total"], r["iterations"], flush=True)
    dump("radial_ref.json", out)


def _capture_stdout(fn):
    """Run fn() with file descriptor 1 redirected; return (result, captured text)."""
    import tempfile
    sys.stdout.flush()
    saved = os.dup(1)
    with tempfile.TemporaryFile(mode="w+b") as tmp:
        os.dup2(tmp.fileno(), 1)
        try:
            res = fn()
        finally:
            sys.stdout.flush()
            os.dup2(saved, 1)
            os.close(saved)
        tmp.seek(0)
        return res, tmp.read().decode(errors="replace")


def _iteration_table(text):
    """The reference's per-iteration table (MolecularSCFHelpers.cpp:264-352):
    [iteration, E, dE, dRho, KS, mixing, seconds]."""
    rows = []
    for line in text.splitlines():
        cells = [c.strip() for c in line.split("|")]
        if len(cells) == 11 and cells[0].isdigit():
            rows.append([int(cells[0]), float(cells[1]), float(cells[2]), float(cells[3]), float(cells[4]),
                         float(cells[5]), float(cells[10])])
    return rows


def scf(cases, fname):
    ref = Ref()
    path = os.path.join(HERE, fname)
    out = json.load(open(path)) if os.path.exists(path) else {}
    for name, (n, b, Z, xyz, charge, mult, kind) in cases.items():
        t = time.time()
        try:
            r, text = _capture_stdout(
                lambda: ref.scf_molecule(n, b, Z, np.asarray(xyz, float).ravel(), charge, mult, kind))
            r.pop("density")
            r["history"] = _iteration_table(text)
            hit = [row[0] for row in r["history"] if row[2] < 1e-6]
            r["first_iteration_abs_de_below_1e-6"] = hit[0] if hit else None
        except RuntimeError as e:  # the reference aborts on some inputs (Davidson cap)
            r = {"error": str(e)}
        r.update({"n": list(n), "bounds": list(b), "Z": Z, "xyz": xyz, "charge": charge, "multiplicity": mult,
                  "functional": "PBE96" if kind == PBE96 else "PZ81", "seconds": time.time() - t})
        out[name] = r
        print(name, r.get("total"), r.get("iterations"), r.get("error"), f"{r['seconds']:.1f}s", flush=True)
        dump(fname, out)


def ops():
    """Operator fixtures: seeded inputs on small grids with the reference's outputs."""
    ref = Ref()
    rng = np.random.default_rng(20261203)
    n = (11, 9, 8)
    b = (-3.0, 3.4, -2.5, 2.9, -2.2, 2.0)
    N = int(np.prod(n))
    x = np.linspace(b[0], b[1], n[0])
    y = np.linspace(b[2], b[3], n[1])
    z = np.linspace(b[4], b[5], n[2])
    Zc, Yc, Xc = np.meshgrid(z, y, x, indexing="ij")
    r2 = Xc ** 2 + Yc ** 2 + Zc ** 2
    na = (0.8 * np.exp(-0.9 * r2) + 1e-3 * rng.random(N).reshape(r2.shape)).ravel()
    nb = (0.5 * np.exp(-0.6 * r2) + 1e-3 * rng.random(N).reshape(r2.shape)).ravel()
    nb[::17] = 0.0  # floored and half-polarised points
    na[::23] = 0.0
    V = rng.standard_normal(N)
    psi = rng.standard_normal((3, N))
    fx = {"n": list(n), "bounds": list(b), "na": na.tolist(), "nb": nb.tolist(), "V": V.tolist(),
          "psi": psi.tolist()}
    fx["hpsi"] = [ref.apply_hamiltonian(n, b, V, p).tolist() for p in psi]
    rho = na + nb
    fx["vh"] = ref.hartree_potential(n, b, rho).tolist()
    fx["eh"] = ref.hartree_energy(n, b, rho, np.asarray(fx["vh"]))
    for kind, tag in ((PZ81, "pz81"), (PBE96, "pbe96")):
        fx[f"vxc_{tag}_a"] = ref.xc_potential(kind, n, b, na, nb, 0).tolist()
        fx[f"vxc_{tag}_b"] = ref.xc_potential(kind, n, b, na, nb, 1).tolist()
        fx[f"exc_{tag}"] = ref.xc_energy(kind, n, b, na, nb)
    fx["T"] = ref.kinetic_energy(n, b, psi, [1, 1, 1])
    fx["dens"] = ref.spin_density(psi, [1, 1, 1]).tolist()
    Zs = [8, 1, 1]
    xyz = np.array([[0.05, 0.07, 0.03], [1.43, 0.07, 1.1], [-1.43, 0.07, 1.1]])
    fx["Zs"] = Zs
    fx["xyz"] = xyz.tolist()
    fx["vext"] = ref.nuclear_potential(n, b, Zs, xyz.ravel()).tolist()
    fx["enn"] = ref.nuclear_repulsion(Zs, xyz.ravel())
    dump("ops_ref.json", fx)


def readme(path=None):
    """The reference's published radial results (README.md:171-241, carbon :413-441), read as text
    from the checkout named by DFT_REFERENCE_DIR (default: the reference mount of the build host)."""
    path = path or os.path.join(os.environ.get("DFT_REFERENCE_DIR", "/root/reference"), "README.md")
    text = open(path, encoding="utf-16").read().splitlines()
    rows = []
    for line in text[170:241]:
        cells = [c.strip() for c in line.split("|")]
        if len(cells) > 5 and cells[1].isdigit():
            rows.append(cells)
    pz, pbe = rows[:30], rows[30:60]
    out = {
        "source": "willandru/DFT README.md:171-202 (PZ81) and :210-241 (PBE96): total energies (Ha) and SCF "
                  "iterations, 2000 radial points, Rmax 30",
        "PZ81": {r[1]: {"symbol": r[2], "iterations": int(r[4]), "total": float(r[5])} for r in pz},
        "PBE96": {r[1]: {"symbol": r[2], "iterations": int(r[4]), "total": float(r[5])} for r in pbe},
        "carbon": {
            "PZ81": {"kinetic": 37.056205462, "external": -86.498033226, "hartree": 17.685104600,
                     "xc": -4.773115917, "total": -36.529839081},
            "PBE96": {"kinetic": 37.503752754, "external": -86.968680315, "hartree": 17.750213488,
                      "xc": -5.128098307, "total": -36.842812379},
            "source": "README.md:413-441",
        },
    }
    dump("readme_radial.json", out)


if __name__ == "__main__":
    what = sys.argv[1:] or ["readme", "radial", "scf_small", "ops"]
    for w in what:
        if w == "readme":
            readme()
        elif w == "radial":
            radial()
        elif w == "scf_small":
            scf(SCF_SMALL, "scf_ref.json")
        elif w == "scf_h2_48":
            scf(SCF_C1, "scf_h2_48_ref.json")
        elif w == "ops":
            ops()
        else:
            raise SystemExit(f"unknown fixture group {w}")
