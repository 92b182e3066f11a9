"""CPU: pin the plain-C oracle (oracle/dft_oracle.c) to the reference.

Two pins: (1) the reference's own published radial results (README tables, committed as
tests/golden/readme_radial.json) and fixtures generated by the reference itself
(tests/golden/*_ref.json, see make_golden.py); (2) where the reference library was built
here (oracle/_ref), live bit-for-bit comparison on seeded inputs.
"""
import numpy as np
import pytest

from conftest import gaussian_density, golden
from oracle.bindings import PBE96, PZ81

GRIDS = [
    ((11, 9, 8), (-3.0, 3.4, -2.5, 2.9, -2.2, 2.0)),
    ((7, 7, 7), (-8.1, 7.9) * 3),
    ((5, 6, 4), (-2.0, 2.2, -1.0, 1.5, -1.7, 1.3)),  # non-exact faces: x_{n-1} != xmax
]


def test_ops_fixture(port):
    fx = golden("ops_ref.json")
    n, b = tuple(fx["n"]), tuple(fx["bounds"])
    na, nb, V = map(np.asarray, (fx["na"], fx["nb"], fx["V"]))
    psi = np.asarray(fx["psi"])
    for p, h in zip(psi, fx["hpsi"]):
        assert np.array_equal(port.apply_hamiltonian(n, b, V, p), np.asarray(h))
    vh = port.hartree_potential(n, b, na + nb)
    assert np.array_equal(vh, np.asarray(fx["vh"]))
    assert port.hartree_energy(n, b, na + nb, vh) == fx["eh"]
    for kind, tag in ((PZ81, "pz81"), (PBE96, "pbe96")):
        assert np.array_equal(port.xc_potential(kind, n, b, na, nb, 0), np.asarray(fx[f"vxc_{tag}_a"]))
        assert np.array_equal(port.xc_potential(kind, n, b, na, nb, 1), np.asarray(fx[f"vxc_{tag}_b"]))
        assert port.xc_energy(kind, n, b, na, nb) == fx[f"exc_{tag}"]
    assert port.kinetic_energy(n, b, psi, [1, 1, 1]) == fx["T"]
    assert np.array_equal(port.spin_density(psi, [1, 1, 1]), np.asarray(fx["dens"]))
    xyz = np.asarray(fx["xyz"]).ravel()
    assert np.array_equal(port.nuclear_potential(n, b, fx["Zs"], xyz), np.asarray(fx["vext"]))
    assert port.nuclear_repulsion(fx["Zs"], xyz) == fx["enn"]


@pytest.mark.parametrize("n,b", GRIDS)
def test_ops_live_bit_exact(port, ref, n, b):
    rng = np.random.default_rng(7)
    N = int(np.prod(n))
    na, nb = gaussian_density(n, b, 3)
    V, psi = rng.standard_normal(N), rng.standard_normal(N)
    assert np.array_equal(port.apply_hamiltonian(n, b, V, psi), ref.apply_hamiltonian(n, b, V, psi))
    assert np.array_equal(port.hartree_potential(n, b, na + nb), ref.hartree_potential(n, b, na + nb))
    for kind in (PZ81, PBE96):
        for s in (0, 1):
            assert np.array_equal(port.xc_potential(kind, n, b, na, nb, s), ref.xc_potential(kind, n, b, na, nb, s))
        assert port.xc_energy(kind, n, b, na, nb) == ref.xc_energy(kind, n, b, na, nb)
    ga, gb = rng.random(N), -rng.random(N)
    for kind in (PZ81, PBE96):
        assert np.array_equal(port.xc_evaluate(kind, na, nb, ga, gb), ref.xc_evaluate(kind, na, nb, ga, gb))


def test_xc_evaluate_edges(port, ref):
    """Floor, full polarisation, zero gradient and sign of the gradient (PBE96.cpp:814-966)."""
    na = np.array([0.0, 1e-21, 1e-20, 0.3, 0.3, 0.0, 2.0, 1e-8, 5.0, 0.1])
    nb = np.array([0.0, 0.0, 1e-21, 0.0, 0.3, 0.4, 1e-30, 1e-8, 5.0, 0.2])
    ga = np.array([0.0, 1.0, 0.0, 0.5, -0.5, 0.0, 3.0, 0.0, -1e3, 0.2])
    gb = np.array([0.0, 0.0, 2.0, 0.0, 0.5, -0.7, 0.0, 1e-9, 1e3, -0.25])
    for kind in (PZ81, PBE96):
        assert np.array_equal(port.xc_evaluate(kind, na, nb, ga, gb), ref.xc_evaluate(kind, na, nb, ga, gb))


def test_davidson_live(port, ref):
    n, b = (11, 9, 8), (-3.0, 3.4, -2.5, 2.9, -2.2, 2.0)
    xyz = np.array([[0.05, 0.07, 0.03], [1.43, 0.07, 1.1], [-1.43, 0.07, 1.1]]).ravel()
    vext = ref.nuclear_potential(n, b, [8, 1, 1], xyz)
    e1, p1 = port.solve_orbitals(n, b, vext, 4)
    e2, p2 = ref.solve_orbitals(n, b, vext, 4)
    assert np.array_equal(e1, e2) and np.array_equal(p1, p2)


def test_radial_vs_readme(port):
    """The oracle reproduces the reference's published energies to the README's print precision."""
    rd = golden("readme_radial.json")
    for fname, kind in (("PZ81", PZ81), ("PBE96", PBE96)):
        for Z in (1, 2, 6, 8, 11, 26):
            r = port.solve_atom(Z, kind)
            assert abs(r["total"] - rd[fname][str(Z)]["total"]) < 5e-8, (fname, Z)
    for fname, kind in (("PZ81", PZ81), ("PBE96", PBE96)):
        r = port.solve_atom(6, kind)
        c = rd["carbon"][fname]
        for k_o, k_r in (("kinetic", "kinetic"), ("external", "external"), ("hartree", "hartree"), ("xc", "xc")):
            assert abs(r[k_o] - c[k_r]) < 5e-9


def test_radial_vs_reference_fixture(port):
    """Bit-for-bit against the reference's own runs (radial_ref.json), a sample of atoms."""
    fx = golden("radial_ref.json")
    for run in fx["runs"]:
        if run["Z"] not in (3, 24, 29):
            continue
        kind = PZ81 if run["functional"] == "PZ81" else PBE96
        r = port.solve_atom(run["Z"], kind)
        assert r["total"] == run["total"]
        assert r["iterations"] == run["iterations"]
        assert r["eigenvalues"] == run["eigenvalues"]


def test_scf_small_vs_reference_fixture(port):
    fx = golden("scf_ref.json")
    for name in ("h2_7_pz81", "h2o_9_pz81", "h3_14_pbe96_doublet", "h2_16_pbe96"):
        c = fx[name]
        kind = PZ81 if c["functional"] == "PZ81" else PBE96
        r = port.scf_molecule(c["n"], c["bounds"], c["Z"], np.ravel(c["xyz"]), c["charge"], c["multiplicity"], kind)
        assert r["total"] == c["total"], name
        assert r["iterations"] == c["iterations"], name


def test_scf_reference_errors(port):
    fx = golden("scf_ref.json")
    c = fx["o2_9_pz81_triplet"]  # the reference aborts: Davidson cap (EigenvalueSolverMolecule.cpp:1214-1220)
    with pytest.raises(RuntimeError, match="no convergio"):
        port.scf_molecule(c["n"], c["bounds"], c["Z"], np.ravel(c["xyz"]), c["charge"], c["multiplicity"], PZ81)
    with pytest.raises(RuntimeError, match="orbitales"):  # zero beta electrons
        port.scf_molecule((7, 7, 7), (-8.1, 7.9) * 3, [1, 1], [-0.7, 0, 0, 0.7, 0, 0], 0, 3, PZ81)
    with pytest.raises(RuntimeError, match="paridad"):
        port.scf_molecule((7, 7, 7), (-8.1, 7.9) * 3, [1, 1], [-0.7, 0, 0, 0.7, 0, 0], 0, 2, PZ81)


def test_atomic_configuration(port, ref):
    for Z in range(1, 31):
        assert port.atomic_configuration(Z) == ref.atomic_configuration(Z)
