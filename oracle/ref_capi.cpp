// Test infrastructure only: a flat extern "C" face over the reference sources
// (willandru/DFT, src/dft/*.cpp), compiled beside them into oracle/_ref/ by
// oracle/Makefile.  The tests load it with ctypes to pin the plain-C restatement
// (oracle/dft_oracle.c) and to produce golden fixtures; nothing in the product
// links it.  Every function forwards to the reference call named in its comment
// and converts C++ exceptions into a non-zero return code with a message.
#include "AtomicDFT.h"
#include "DFTConstants.h"
#include "CartesianGrid.h"
#include "DFTData.h"
#include "EigenvalueSolver.h"
#include "EigenvalueSolverMolecule.h"
#include "ElectronDensityMolecule.h"
#include "ElectronicConfiguration.h"
#include "ExchangeCorrelation.h"
#include "ExchangeCorrelationMolecule.h"
#include "HartreePotential.h"
#include "HartreePotentialMolecule.h"
#include "KohnShamHamiltonian.h"
#include "KohnShamHamiltonianMolecule.h"
#include "MolecularSCFHelpers.h"
#include "MolecularSCFIteration.h"
#include "Molecule.h"
#include "NuclearPotential.h"
#include "NuclearRepulsion.h"
#include "PBE96.h"
#include "PZ81.h"
#include "RadialGrid.h"
#include "SelfConsistentFieldMolecule.h"
#include "TotalEnergy.h"
#include "TotalEnergyMolecule.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

const XCFunctional& functional(int kind) {
    static PZ81 pz;
    static PBE96 pbe;
    return kind == 1 ? static_cast<const XCFunctional&>(pbe)
                     : static_cast<const XCFunctional&>(pz);
}

CartesianGrid grid_of(const long* n, const double* b) {
    return CartesianGrid(n[0], n[1], n[2], b[0], b[1], b[2], b[3], b[4], b[5]);
}

std::vector<double> vec(const double* p, size_t n) {
    return std::vector<double>(p, p + n);
}

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

Molecule molecule_of(int nnuc, const int* Z, const double* xyz, int charge) {
    Molecule m(charge);
    for (int a = 0; a < nnuc; ++a) m.addNucleus(Z[a], xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2]);
    return m;
}

void copy_out(const std::vector<double>& v, double* out) {
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// XCFunctional::evaluate (XCFunctional.h:15-22; PZ81.cpp:437, PBE96.cpp:814), vectorised over m points.
int ref_xc_evaluate(int kind, long m, const double* na, const double* nb, const double* ga,
                    const double* gb, double* out5) {
    return guard([&] {
        const XCFunctional& f = functional(kind);
        for (long i = 0; i < m; ++i) {
            XCResult r = f.evaluate(XCInput{na[i], nb[i], ga[i], gb[i]});
            out5[5 * i + 0] = r.energyPerElectron;
            out5[5 * i + 1] = r.potentialAlpha;
            out5[5 * i + 2] = r.potentialBeta;
            out5[5 * i + 3] = r.gradientCoefficientAlpha;
            out5[5 * i + 4] = r.gradientCoefficientBeta;
        }
    });
}

// applyMolecularKohnShamHamiltonian (KohnShamHamiltonianMolecule.cpp:7-183)
int ref_apply_hamiltonian(const long* n, const double* b, const double* V, const double* psi, double* out) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        copy_out(applyMolecularKohnShamHamiltonian(g, vec(V, g.getSize()), vec(psi, g.getSize())), out);
    });
}

// calculateHartreePotential (HartreePotentialMolecule.cpp:99-324)
int ref_hartree_potential(const long* n, const double* b, const double* rho, double* out) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        copy_out(calculateHartreePotential(g, vec(rho, g.getSize())), out);
    });
}

// calculateHartreeEnergy (HartreePotentialMolecule.cpp:326-379)
int ref_hartree_energy(const long* n, const double* b, const double* rho, const double* vh, double* e) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        *e = calculateHartreeEnergy(g, vec(rho, g.getSize()), vec(vh, g.getSize()));
    });
}

// calculateMolecularSpinExchangeCorrelationPotential (ExchangeCorrelationMolecule.cpp:576-747)
int ref_xc_potential(int kind, const long* n, const double* b, const double* na, const double* nb, int spin,
                     double* out) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        copy_out(calculateMolecularSpinExchangeCorrelationPotential(functional(kind), g, vec(na, g.getSize()),
                                                                     vec(nb, g.getSize()), spin),
                 out);
    });
}

// calculateMolecularExchangeCorrelationEnergy (ExchangeCorrelationMolecule.cpp:749-842)
int ref_xc_energy(int kind, const long* n, const double* b, const double* na, const double* nb, double* e) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        *e = calculateMolecularExchangeCorrelationEnergy(functional(kind), g, vec(na, g.getSize()),
                                                         vec(nb, g.getSize()));
    });
}

// NuclearPotential::calculate (NuclearPotential.cpp:6-34)
int ref_nuclear_potential(const long* n, const double* b, int nnuc, const int* Z, const double* xyz,
                          double* out) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        copy_out(NuclearPotential::calculate(molecule_of(nnuc, Z, xyz, 0), g), out);
    });
}

// NuclearRepulsion::calculate (NuclearRepulsion.cpp:6-54)
int ref_nuclear_repulsion(int nnuc, const int* Z, const double* xyz, double* e) {
    return guard([&] { *e = NuclearRepulsion::calculate(molecule_of(nnuc, Z, xyz, 0)); });
}

// calculateMolecularKineticEnergy (TotalEnergyMolecule.cpp:13-199); psi is nb x N band-major.
int ref_kinetic_energy(const long* n, const double* b, int nbands, const double* psi, const int* electrons,
                       double* e) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        std::vector<MolecularOrbital> orbs(nbands);
        for (int i = 0; i < nbands; ++i) {
            orbs[i].electrons = electrons[i];
            orbs[i].psi = vec(psi + (size_t)i * g.getSize(), g.getSize());
        }
        *e = calculateMolecularKineticEnergy(g, orbs);
    });
}

// calculateMolecularSpinDensity (ElectronDensityMolecule.cpp:5-76)
int ref_spin_density(long N, int nbands, const double* psi, const int* electrons, double* out) {
    return guard([&] {
        std::vector<MolecularOrbital> orbs(nbands);
        for (int i = 0; i < nbands; ++i) {
            orbs[i].electrons = electrons[i];
            orbs[i].spin = SpinChannel::Alpha;
            orbs[i].psi = vec(psi + (size_t)i * N, N);
        }
        copy_out(calculateMolecularSpinDensity(orbs, SpinChannel::Alpha), out);
    });
}

// solveMolecularOrbitals (EigenvalueSolverMolecule.cpp:1233-1300).  init may be NULL.
int ref_solve_orbitals(const long* n, const double* b, const double* V, int norb, const double* init,
                       double* psi_out, double* eig_out) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        std::vector<MolecularOrbital> guess;
        if (init) {
            guess.resize(norb);
            for (int i = 0; i < norb; ++i) guess[i].psi = vec(init + (size_t)i * g.getSize(), g.getSize());
        }
        std::vector<int> occ(norb, 1);
        auto orbs = solveMolecularOrbitals(g, vec(V, g.getSize()), norb, occ, SpinChannel::Alpha, guess);
        for (int i = 0; i < norb; ++i) {
            eig_out[i] = orbs[i].eigenvalue;
            std::memcpy(psi_out + (size_t)i * g.getSize(), orbs[i].psi.data(), g.getSize() * sizeof(double));
        }
    });
}

// solveMolecularSelfConsistentField (SelfConsistentFieldMolecule.cpp:50-561).
// energies6 = {kinetic, external, hartree, xc, nuclearRepulsion, total};
// stats4 = {iterations, converged, densityDifference, maxKSResidual}; eig_out holds the alpha
// then beta eigenvalues (capacity n_eig); dens_out (optional) holds n_alpha then n_beta.
int ref_scf_molecule(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int charge,
                     int multiplicity, int kind, double* energies6, double* stats4, int n_eig, double* eig_out,
                     double* dens_out) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        Molecule m = molecule_of(nnuc, Z, xyz, charge);
        MolecularResult r = solveMolecularSelfConsistentField(g, m, charge, multiplicity, functional(kind));
        const EnergyComponents& e = r.scf.energy;
        energies6[0] = e.kinetic;
        energies6[1] = e.external;
        energies6[2] = e.hartree;
        energies6[3] = e.exchangeCorrelation;
        energies6[4] = e.nuclearRepulsion;
        energies6[5] = e.total;
        stats4[0] = r.scf.iterations;
        stats4[1] = r.scf.converged ? 1.0 : 0.0;
        stats4[2] = r.scf.densityDifference;
        stats4[3] = r.scf.maxKSResidual;
        int k = 0;
        for (const auto& o : r.scf.molecularOrbitals)
            if (k < n_eig) eig_out[k++] = o.eigenvalue;
        if (dens_out) {
            copy_out(r.scf.alphaDensity, dens_out);
            copy_out(r.scf.betaDensity, dens_out + g.getSize());
        }
    });
}

// A bounded CPU-baseline sample of the molecular SCF: buildInitialMolecularDensities
// (MolecularSCFHelpers.cpp:515-579) then `iterations` calls of executeMolecularSCFIteration
// (MolecularSCFIteration.cpp:12-252) with the reference's linear mixing at 0.25.
// seconds2 = {initialisation seconds, seconds per iteration (mean)}.
int ref_scf_sample(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int multiplicity,
                   int kind, int iterations, double* seconds2) {
    return guard([&] {
        CartesianGrid g = grid_of(n, b);
        Molecule m = molecule_of(nnuc, Z, xyz, 0);
        int ne = 0;
        for (int a = 0; a < nnuc; ++a) ne += Z[a];
        const int sd = multiplicity - 1;
        const int na = (ne + sd) / 2, nbeta = (ne - sd) / 2;
        const bool closed = multiplicity == 1;
        auto t0 = std::chrono::steady_clock::now();
        std::vector<double> vext = NuclearPotential::calculate(m, g);
        std::vector<double> da, db;
        std::vector<MolecularOrbital> pa, pb;
        buildInitialMolecularDensities(g, m, na, nbeta, closed, da, db, pa, pb);
        auto t1 = std::chrono::steady_clock::now();
        for (int it = 0; it < iterations; ++it) {
            MolecularSCFIterationResult r =
                executeMolecularSCFIteration(g, m, functional(kind), vext, da, db, na, nbeta, closed, pa, pb);
            mixDensity(da, r.outputAlphaDensity, 0.25);
            mixDensity(db, r.outputBetaDensity, 0.25);
            pa = r.alphaOrbitals;
            if (!closed) pb = r.betaOrbitals;
        }
        auto t2 = std::chrono::steady_clock::now();
        seconds2[0] = std::chrono::duration<double>(t1 - t0).count();
        seconds2[1] = std::chrono::duration<double>(t2 - t1).count() / std::max(iterations, 1);
    });
}

// The reference's molecular SCF loop (SelfConsistentFieldMolecule.cpp:180-500) run until the
// benchmark metric's stop |E_k - E_{k-1}| < de_stop (or the reference's own three-criterion
// stop, or max_iterations): buildInitialMolecularDensities, then executeMolecularSCFIteration
// with the loop's adaptive mixing (constants :27-31, pre-update factor applied, :447-484) and
// its orbital carry-over (:402-409).  out5 = {seconds in total, initialisation seconds,
// iterations, final total energy, |dE| of the last iteration}.
int ref_scf_to_de(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int multiplicity,
                  int kind, double de_stop, int max_iterations, double* out5) {
    return guard([&] {
        constexpr double MIN_MIXING = 0.10, MAX_MIXING = 0.50, MIXING_INCREASE = 1.10, MIXING_DECREASE = 0.75,
                         OSCILLATION_FACTOR = 1.05;
        const auto t0 = std::chrono::steady_clock::now();
        CartesianGrid g = grid_of(n, b);
        Molecule m = molecule_of(nnuc, Z, xyz, 0);
        int ne = 0;
        for (int a = 0; a < nnuc; ++a) ne += Z[a];
        const int sd = multiplicity - 1;
        const int na = (ne + sd) / 2, nbeta = (ne - sd) / 2;
        const bool closed = multiplicity == 1;
        std::vector<double> vext = NuclearPotential::calculate(m, g);
        std::vector<double> da, db;
        std::vector<MolecularOrbital> pa, pb;
        buildInitialMolecularDensities(g, m, na, nbeta, closed, da, db, pa, pb);
        const auto t1 = std::chrono::steady_clock::now();
        double prevE = std::numeric_limits<double>::infinity(), prevD = prevE, mixing = 0.25, dE = prevE, E = 0.0;
        int it = 0;
        for (it = 1; it <= max_iterations; ++it) {
            const double imix = mixing;
            MolecularSCFIterationResult r =
                executeMolecularSCFIteration(g, m, functional(kind), vext, da, db, na, nbeta, closed, pa, pb);
            E = r.energy.total;
            dE = std::isfinite(prevE) ? std::fabs(E - prevE) : std::numeric_limits<double>::infinity();
            const bool conv = dE < DFTConstants::ENERGY_TOL &&
                              r.effectiveDensityDifference < DFTConstants::DENSITY_TOL &&
                              r.residual < DFTConstants::KS_RESIDUAL_TOL;
            if (conv || dE < de_stop) break;
            pa = r.alphaOrbitals;
            if (!closed) pb = r.betaOrbitals;
            if (std::isfinite(prevD)) {
                if (r.effectiveDensityDifference > prevD * OSCILLATION_FACTOR)
                    mixing = std::max(MIN_MIXING, mixing * MIXING_DECREASE);
                else if (r.effectiveDensityDifference < prevD)
                    mixing = std::min(MAX_MIXING, mixing * MIXING_INCREASE);
            }
            mixDensity(da, r.outputAlphaDensity, imix);
            mixDensity(db, r.outputBetaDensity, imix);
            prevD = r.effectiveDensityDifference;
            prevE = E;
        }
        const auto t2 = std::chrono::steady_clock::now();
        out5[0] = std::chrono::duration<double>(t2 - t0).count();
        out5[1] = std::chrono::duration<double>(t1 - t0).count();
        out5[2] = std::min(it, max_iterations);
        out5[3] = E;
        out5[4] = dE;
    });
}

// solveAtom (AtomicDFT.cpp:7-42) with getAtomicConfiguration(Z) (ElectronicConfiguration.cpp:49-146).
// energies5 = {kinetic, external, hartree, xc, total}; stats4 = {iterations, converged, dRho, KS};
// eig_out: eigenvalues in the reference's orbital order (alpha states then beta states).
int ref_solve_atom(int Z, int kind, long points, double rmax, double* energies5, double* stats4, int n_eig,
                   double* eig_out, int* n_eig_written) {
    return guard([&] {
        RadialGrid grid(points, rmax);
        AtomicResult r = solveAtom(grid, getAtomicConfiguration(Z), functional(kind));
        const EnergyComponents& e = r.scf.energy;
        energies5[0] = e.kinetic;
        energies5[1] = e.external;
        energies5[2] = e.hartree;
        energies5[3] = e.exchangeCorrelation;
        energies5[4] = e.total;
        stats4[0] = r.scf.iterations;
        stats4[1] = r.scf.converged ? 1.0 : 0.0;
        stats4[2] = r.scf.densityDifference;
        stats4[3] = r.scf.maxKSResidual;
        int k = 0;
        for (const auto& o : r.scf.orbitals)
            if (k < n_eig) eig_out[k++] = o.eigenvalue;
        *n_eig_written = k;
    });
}

// Radial operators on RadialGrid(points, rmax).r:
// calculateHartreePotential (HartreePotential.cpp:8-86)
int ref_radial_hartree(long points, double rmax, const double* rho, double* out) {
    return guard([&] {
        RadialGrid grid(points, rmax);
        copy_out(calculateHartreePotential(grid.coordinates(), vec(rho, points)), out);
    });
}

// calculateSpinExchangeCorrelationPotential (ExchangeCorrelation.cpp:154-274)
int ref_radial_xc_potential(int kind, long points, double rmax, const double* na, const double* nb, int spin,
                            double* out) {
    return guard([&] {
        RadialGrid grid(points, rmax);
        copy_out(calculateSpinExchangeCorrelationPotential(functional(kind), grid.coordinates(), vec(na, points),
                                                           vec(nb, points), spin),
                 out);
    });
}

// calculateSpinExchangeCorrelationEnergy (ExchangeCorrelation.cpp:276-371)
int ref_radial_xc_energy(int kind, long points, double rmax, const double* na, const double* nb, double* e) {
    return guard([&] {
        RadialGrid grid(points, rmax);
        *e = calculateSpinExchangeCorrelationEnergy(functional(kind), grid.coordinates(), vec(na, points),
                                                    vec(nb, points));
    });
}

// buildKohnShamHamiltonian (KohnShamHamiltonian.cpp:6-101) + solveOrbital (EigenvalueSolver.cpp:323-404)
int ref_radial_solve_orbital(long points, double rmax, const double* veff, int l, int index, double* eig,
                             double* u_out) {
    return guard([&] {
        RadialGrid grid(points, rmax);
        TridiagonalMatrix h = buildKohnShamHamiltonian(grid.coordinates(), vec(veff, points), l);
        AtomicOrbital o = solveOrbital(h, grid.coordinates(), 1, l, 1, index);
        *eig = o.eigenvalue;
        copy_out(o.u, u_out);
    });
}

// countEigenvaluesBelow (EigenvalueSolver.cpp:37-92) on the radial Hamiltonian.
int ref_radial_sturm_count(long points, double rmax, const double* veff, int l, double energy, long* count) {
    return guard([&] {
        RadialGrid grid(points, rmax);
        TridiagonalMatrix h = buildKohnShamHamiltonian(grid.coordinates(), vec(veff, points), l);
        *count = (long)countEigenvaluesBelow(h, energy);
    });
}

// getAtomicConfiguration (ElectronicConfiguration.cpp:49-146): rows of {n, l, alpha, beta}.
int ref_atomic_configuration(int Z, int cap, int* rows, int* nrows) {
    return guard([&] {
        AtomicConfiguration c = getAtomicConfiguration(Z);
        int k = 0;
        for (const auto& s : c.states) {
            if (k < cap) {
                rows[4 * k + 0] = s.n;
                rows[4 * k + 1] = s.l;
                rows[4 * k + 2] = s.alphaElectrons;
                rows[4 * k + 3] = s.betaElectrons;
            }
            ++k;
        }
        *nrows = k;
    });
}

}  // extern "C"
