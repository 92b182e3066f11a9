// Reference-side integration check: the reference's own types and CPU functions linked in
// one program with the dft_b200.hpp drop-in.  Each call is made twice, once through the
// reference (global namespace) and once through dftb200::, and the results compared.
// Built by `make -C oracle shim` where the reference tree is present; run by
// tests/test_gpu_shim.py on a GPU.  Exit code 0 = all comparisons within tolerance.
#include <cmath>
#include <cstdio>
#include <vector>

#include "AtomicDFT.h"
#include "HartreePotentialMolecule.h"
#include "KohnShamHamiltonianMolecule.h"
#include "SelfConsistentFieldMolecule.h"
#include "dft_b200.hpp"

static int failures = 0;

static void expect(bool ok, const char* what, double a, double b) {
    std::printf("%-44s cpu=% .12f gpu=% .12f  %s\n", what, a, b, ok ? "ok" : "MISMATCH");
    if (!ok) ++failures;
}

int main() {
    PZ81 pz81;
    PBE96 pbe96;

    // H psi and Poisson on a small grid: bit-identical
    CartesianGrid g(9, 8, 7, -3.0, 3.0, -2.5, 2.5, -2.0, 2.0);
    std::vector<double> V(g.getSize()), psi(g.getSize()), rho(g.getSize());
    for (std::size_t i = 0; i < g.getSize(); ++i) {
        V[i] = std::sin(0.37 * i);
        psi[i] = std::cos(0.11 * i * i);
        rho[i] = std::exp(-0.01 * (double)((i * 7) % 101));
    }
    auto h_cpu = applyMolecularKohnShamHamiltonian(g, V, psi);
    auto h_gpu = dftb200::applyMolecularKohnShamHamiltonian(g, V, psi);
    expect(h_cpu == h_gpu, "applyMolecularKohnShamHamiltonian (bitwise)", h_cpu[17], h_gpu[17]);
    auto v_cpu = calculateHartreePotential(g, rho);
    auto v_gpu = dftb200::calculateHartreePotential(g, rho);
    expect(v_cpu == v_gpu, "calculateHartreePotential (bitwise)", v_cpu[100], v_gpu[100]);

    // the reference demo's H2 (main.cpp:74-117)
    Molecule h2(0);
    h2.addNucleus(1, -0.7, 0.0, 0.0);
    h2.addNucleus(1, 0.7, 0.0, 0.0);
    CartesianGrid h2g(7, 7, 7, -8.1, 7.9, -8.1, 7.9, -8.1, 7.9);
    MolecularResult a = solveMolecularSelfConsistentField(h2g, h2, 0, 1, pz81);
    MolecularResult b = dftb200::solveMolecularSelfConsistentField(h2g, h2, 0, 1, pz81);
    expect(std::fabs(a.scf.energy.total - b.scf.energy.total) < 1e-7 && b.scf.converged,
           "solveMolecularSelfConsistentField H2 7^3", a.scf.energy.total, b.scf.energy.total);

    // radial carbon, both functionals
    RadialGrid rg(2000, 30.0);
    for (const XCFunctional* f : {(const XCFunctional*)&pz81, (const XCFunctional*)&pbe96}) {
        AtomicResult ra = solveAtom(rg, getAtomicConfiguration(6), *f);
        AtomicResult rb = dftb200::solveAtom(rg, getAtomicConfiguration(6), *f);
        expect(std::fabs(ra.scf.energy.total - rb.scf.energy.total) < 1e-9 && rb.scf.converged,
               f == &pz81 ? "solveAtom C PZ81" : "solveAtom C PBE96", ra.scf.energy.total, rb.scf.energy.total);
    }
    std::printf("%s\n", failures ? "FAILED" : "all ok");
    return failures ? 1 : 0;
}
