// dft_b200.hpp — header-only C++ drop-in for the reference's driver API (willandru/DFT).
//
// Include it from code built against the reference's headers (CartesianGrid.h, Molecule.h,
// RadialGrid.h, DFTData.h, XCFunctional.h, PZ81.h, PBE96.h must be on the include path)
// and link libdft_b200.so.  Every function has the reference's signature and semantics
// and lives in namespace dftb200, so a caller switches with a namespace qualifier or a
// using-declaration:
//
//     #include "dft_b200.hpp"
//     using dftb200::solveMolecularSelfConsistentField;   // instead of the CPU one
//
// Host std::vector inputs are copied to the GPU and results copied back; failures are
// rethrown as the reference's exception types (std::invalid_argument for bad input,
// std::runtime_error otherwise).  One process-wide context on device 0 (override with
// dftb200::set_device before the first call).
#pragma once

#include <algorithm>
#include <memory>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

#include "dft_b200.h"

#include "CartesianGrid.h"
#include "DFTData.h"
#include "ElectronicConfiguration.h"
#include "Molecule.h"
#include "PBE96.h"
#include "PZ81.h"
#include "RadialGrid.h"
#include "XCFunctional.h"

namespace dftb200 {

namespace detail {

inline void check(dft_status_t s) {
    if (s == DFT_OK) return;
    const std::string msg = dft_last_error_message();
    if (s == DFT_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

inline int& device_index() {
    static int d = 0;
    return d;
}

struct Ctx {
    dft_context* c = nullptr;
    Ctx() { check(dft_context_create(device_index(), &c)); }
    ~Ctx() { dft_context_destroy(c); }
};

inline dft_context* ctx() {
    static Ctx instance;
    return instance.c;
}

// the reference selects the functional by dynamic type (XCFunctional.h:15-22)
inline dft_xc_kind kind_of(const XCFunctional& f) {
    if (dynamic_cast<const PBE96*>(&f)) return DFT_XC_PBE96;
    if (dynamic_cast<const PZ81*>(&f)) return DFT_XC_PZ81;
    throw std::invalid_argument(std::string("unsupported XCFunctional: ") + typeid(f).name());
}

inline dft_grid grid_of(const CartesianGrid& g) {
    return dft_grid{(long)g.getNx(), (long)g.getNy(), (long)g.getNz(), g.getXMin(), g.getXMax(),
                    g.getYMin(),     g.getYMax(),     g.getZMin(),     g.getZMax()};
}

// device buffer owned for the duration of one call
struct Dev {
    void* p = nullptr;
    explicit Dev(size_t bytes) { check(dft_device_alloc(ctx(), bytes, &p)); }
    Dev(const std::vector<double>& h) : Dev(h.size() * sizeof(double)) {
        if (!h.empty()) check(dft_copy_h2d(ctx(), p, h.data(), h.size() * sizeof(double)));
    }
    ~Dev() { dft_device_free(ctx(), p); }
    double* d() const { return static_cast<double*>(p); }
    std::vector<double> get(size_t n) const {
        std::vector<double> h(n);
        if (n) check(dft_copy_d2h(ctx(), h.data(), p, n * sizeof(double)));
        return h;
    }
};

inline void need_size(const CartesianGrid& g, const std::vector<double>& v, const char* what) {
    if (v.size() != g.getSize()) throw std::invalid_argument(what);
}

}  // namespace detail

inline void set_device(int device) { detail::device_index() = device; }

// applyMolecularKohnShamHamiltonian (KohnShamHamiltonianMolecule.h:7-11)
inline std::vector<double> applyMolecularKohnShamHamiltonian(const CartesianGrid& grid,
                                                             const std::vector<double>& effectivePotential,
                                                             const std::vector<double>& psi) {
    detail::need_size(grid, effectivePotential, "El potencial efectivo y la malla cartesiana deben tener el mismo tamano.");
    detail::need_size(grid, psi, "La funcion de onda y la malla cartesiana deben tener el mismo tamano.");
    const dft_grid g = detail::grid_of(grid);
    detail::Dev V(effectivePotential), P(psi), H(psi.size() * sizeof(double));
    detail::check(dft_apply_hamiltonian_dev(detail::ctx(), &g, V.d(), P.d(), H.d(), 1, (long)psi.size()));
    return H.get(psi.size());
}

// calculateHartreePotential (HartreePotentialMolecule.h:7-10)
inline std::vector<double> calculateHartreePotential(const CartesianGrid& grid, const std::vector<double>& density) {
    detail::need_size(grid, density, "La densidad molecular y la malla cartesiana deben tener el mismo tamano.");
    const dft_grid g = detail::grid_of(grid);
    detail::Dev R(density), V(density.size() * sizeof(double));
    detail::check(dft_hartree_dev(detail::ctx(), &g, R.d(), V.d(), 1.0e-8, 10000, nullptr, nullptr));
    return V.get(density.size());
}

// calculateHartreeEnergy (HartreePotentialMolecule.h:12-15)
inline double calculateHartreeEnergy(const CartesianGrid& grid, const std::vector<double>& density,
                                     const std::vector<double>& hartreePotential) {
    detail::need_size(grid, density, "La densidad, el potencial de Hartree y la malla deben tener el mismo tamano.");
    detail::need_size(grid, hartreePotential, "La densidad, el potencial de Hartree y la malla deben tener el mismo tamano.");
    const dft_grid g = detail::grid_of(grid);
    detail::Dev R(density), V(hartreePotential);
    double e = 0.0;
    detail::check(dft_hartree_energy_dev(detail::ctx(), &g, R.d(), V.d(), &e));
    return e;
}

// calculateMolecularSpinExchangeCorrelationPotential (ExchangeCorrelationMolecule.h:8-14)
inline std::vector<double> calculateMolecularSpinExchangeCorrelationPotential(const XCFunctional& functional,
                                                                              const CartesianGrid& grid,
                                                                              const std::vector<double>& alphaDensity,
                                                                              const std::vector<double>& betaDensity,
                                                                              int spin) {
    if (spin != 0 && spin != 1) throw std::invalid_argument("El canal de spin debe ser 0 (alpha) o 1 (beta).");
    detail::need_size(grid, alphaDensity, "La malla cartesiana y las densidades spin deben tener el mismo tamano.");
    detail::need_size(grid, betaDensity, "La malla cartesiana y las densidades spin deben tener el mismo tamano.");
    const dft_grid g = detail::grid_of(grid);
    detail::Dev A(alphaDensity), B(betaDensity), V(alphaDensity.size() * sizeof(double));
    detail::check(dft_xc_dev(detail::ctx(), &g, detail::kind_of(functional), A.d(), B.d(), spin == 0 ? V.d() : nullptr,
                             spin == 1 ? V.d() : nullptr, nullptr));
    return V.get(alphaDensity.size());
}

// calculateMolecularExchangeCorrelationEnergy (ExchangeCorrelationMolecule.h:16-21)
inline double calculateMolecularExchangeCorrelationEnergy(const XCFunctional& functional, const CartesianGrid& grid,
                                                          const std::vector<double>& alphaDensity,
                                                          const std::vector<double>& betaDensity) {
    detail::need_size(grid, alphaDensity, "La malla cartesiana y las densidades spin deben tener el mismo tamano.");
    detail::need_size(grid, betaDensity, "La malla cartesiana y las densidades spin deben tener el mismo tamano.");
    const dft_grid g = detail::grid_of(grid);
    detail::Dev A(alphaDensity), B(betaDensity);
    double e = 0.0;
    detail::check(dft_xc_dev(detail::ctx(), &g, detail::kind_of(functional), A.d(), B.d(), nullptr, nullptr, &e));
    return e;
}

// solveMolecularOrbitals (EigenvalueSolverMolecule.h:20-28): block Davidson over the
// requested orbitals plus three buffer bands; maxIterations caps block iterations.
inline std::vector<MolecularOrbital> solveMolecularOrbitals(const CartesianGrid& grid,
                                                            const std::vector<double>& effectivePotential,
                                                            std::size_t numberOfOrbitals,
                                                            const std::vector<int>& occupations, SpinChannel spin,
                                                            const std::vector<MolecularOrbital>& initialOrbitals = {},
                                                            std::size_t maxIterations = 5000) {
    if (numberOfOrbitals == 0) throw std::invalid_argument("El numero de orbitales debe ser mayor que cero.");
    if (occupations.size() != numberOfOrbitals)
        throw std::invalid_argument("Las ocupaciones no coinciden con el numero de orbitales.");
    if (!initialOrbitals.empty() && initialOrbitals.size() != numberOfOrbitals)
        throw std::invalid_argument("Los orbitales iniciales no coinciden con el numero solicitado.");
    detail::need_size(grid, effectivePotential, "El potencial y la malla no coinciden.");
    const size_t N = grid.getSize();
    const int nb = (int)std::min<size_t>(numberOfOrbitals + 3, N);
    std::vector<double> block((size_t)nb * N, 0.0);
    for (size_t i = 0; i < initialOrbitals.size(); ++i)
        if (initialOrbitals[i].psi.size() == N) std::copy(initialOrbitals[i].psi.begin(), initialOrbitals[i].psi.end(),
                                                          block.begin() + i * N);
    const dft_grid g = detail::grid_of(grid);
    detail::Dev V(effectivePotential), P(block);
    std::vector<double> eig(nb);
    dft_eig_opts o{1.0e-7, (int)std::min<std::size_t>(maxIterations, 1000000), 3, 0, 4};
    detail::check(dft_solve_orbitals_dev(detail::ctx(), &g, V.d(), (int)numberOfOrbitals, nb, P.d(), (long)N,
                                         initialOrbitals.empty() ? 0 : 1, eig.data(), &o, nullptr));
    const std::vector<double> psi = P.get((size_t)nb * N);
    std::vector<MolecularOrbital> out(numberOfOrbitals);
    for (size_t i = 0; i < numberOfOrbitals; ++i) {
        out[i].spin = spin;
        out[i].electrons = occupations[i];
        out[i].eigenvalue = eig[i];
        out[i].psi.assign(psi.begin() + i * N, psi.begin() + (i + 1) * N);
    }
    return out;
}

// solveMolecularSelfConsistentField (SelfConsistentFieldMolecule.h:8-14)
inline MolecularResult solveMolecularSelfConsistentField(const CartesianGrid& grid, const Molecule& molecule,
                                                         int charge, int multiplicity,
                                                         const XCFunctional& functional) {
    const dft_grid g = detail::grid_of(grid);
    std::vector<int> Z;
    std::vector<double> xyz;
    for (const auto& n : molecule.getNuclei()) {
        Z.push_back(n.atomicNumber);
        xyz.insert(xyz.end(), n.position.begin(), n.position.end());
    }
    if (Z.empty()) throw std::invalid_argument("La molecula debe contener al menos un nucleo.");
    int nuclear = 0;
    for (int z : Z) nuclear += z;
    const size_t N = grid.getSize();
    const int ne = std::max(nuclear - charge, 1);
    std::vector<double> eig((size_t)ne + 2), da(N), db(N), va(N), vb(N), orb((size_t)ne * N);
    dft_scf_opts opts;
    dft_scf_default_options(&opts);
    dft_scf_result r{};
    r.eigenvalues = eig.data();
    r.alpha_density = da.data();
    r.beta_density = db.data();
    r.alpha_potential = va.data();
    r.beta_potential = vb.data();
    r.orbitals = orb.data();
    detail::check(dft_scf_molecule(detail::ctx(), &g, (int)Z.size(), Z.data(), xyz.data(), charge, multiplicity,
                                   detail::kind_of(functional), &opts, &r));
    MolecularResult out;
    out.electrons = nuclear - charge;
    out.charge = charge;
    SCFResult& s = out.scf;
    s.energy.kinetic = r.kinetic;
    s.energy.external = r.external;
    s.energy.hartree = r.hartree;
    s.energy.exchangeCorrelation = r.exchange_correlation;
    s.energy.nuclearRepulsion = r.nuclear_repulsion;
    s.energy.total = r.total;
    s.iterations = r.iterations;
    s.converged = r.converged != 0;
    s.densityDifference = r.density_difference;
    s.energyDifference = r.energy_difference;
    s.maxKSResidual = r.max_ks_residual;
    s.alphaDensity = da;
    s.betaDensity = db;
    s.density.resize(N);
    for (size_t i = 0; i < N; ++i) s.density[i] = da[i] + db[i];
    s.alphaEffectivePotential = va;
    s.betaEffectivePotential = vb;
    s.effectivePotential = va;
    for (int i = 0; i < r.n_alpha + r.n_beta; ++i) {
        MolecularOrbital o;
        o.spin = i < r.n_alpha ? SpinChannel::Alpha : SpinChannel::Beta;
        o.electrons = 1;
        o.eigenvalue = eig[i];
        o.psi.assign(orb.begin() + (size_t)i * N, orb.begin() + (size_t)(i + 1) * N);
        s.molecularOrbitals.push_back(std::move(o));
    }
    return out;
}

// solveAtom (AtomicDFT.h:7-11).  Orbital eigenvalues and quantum numbers are returned;
// radial wavefunctions stay on the device.
inline AtomicResult solveAtom(const RadialGrid& grid, const AtomicConfiguration& configuration,
                              const XCFunctional& functional) {
    if (configuration.Z <= 0) throw std::invalid_argument("El numero atomico debe ser mayor que cero.");
    int z = configuration.Z, k = (int)detail::kind_of(functional);
    dft_atom_result r{};
    detail::check(dft_solve_atoms(detail::ctx(), 1, &z, &k, (long)grid.size(), grid.rMax(), &r));
    if (r.status != DFT_OK) throw std::runtime_error("radial SCF failed");
    AtomicResult out;
    out.Z = configuration.Z;
    out.symbol = configuration.symbol;
    for (const auto& st : configuration.states) out.electrons += st.alphaElectrons + st.betaElectrons;
    SCFResult& s = out.scf;
    s.energy.kinetic = r.kinetic;
    s.energy.external = r.external;
    s.energy.hartree = r.hartree;
    s.energy.exchangeCorrelation = r.exchange_correlation;
    s.energy.total = r.total;
    s.iterations = r.iterations;
    s.converged = r.converged != 0;
    s.densityDifference = r.density_difference;
    s.maxKSResidual = r.max_ks_residual;
    int q = 0;
    for (int spin = 0; spin < 2; ++spin)
        for (const auto& st : configuration.states) {
            const int e = spin == 0 ? st.alphaElectrons : st.betaElectrons;
            if (e <= 0 || q >= r.n_orbitals) continue;
            AtomicOrbital o;
            o.n = st.n;
            o.l = st.l;
            o.spin = spin == 0 ? SpinChannel::Alpha : SpinChannel::Beta;
            o.electrons = e;
            o.eigenvalue = r.eigenvalues[q++];
            s.orbitals.push_back(std::move(o));
        }
    return out;
}

}  // namespace dftb200
