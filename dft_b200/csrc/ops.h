// Internal (C++) interface of the dft_b200 device operators.  The extern "C" layer in
// capi.cu validates arguments, catches dftb::Error and forwards here.  All pointers are
// device pointers; every function is stream-ordered on ctx->stream unless it returns a
// host scalar, in which case it synchronises.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include <array>
#include <vector>

#include "common.cuh"

namespace dftb {

// cuTensorMapEncodeTiled (driver entry point looked up once; nullptr when unavailable)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// H psi over a band block (bit-identical to the reference per band).
// hpsi_tma_eligible: whether the TMA plane-ring variant takes this grid and block.
bool hpsi_tma_eligible(const Grid& g, const double* psi, long long ld);
void apply_hamiltonian(dft_context* ctx, const Grid& g, const double* V, const double* psi, double* hpsi, int nbands,
                       long long ld);

// Jacobi Poisson with the reference's stopping rule.  Returns the sweep count.
struct JacobiResult {
    long sweeps;
    double last_diff;
};
// guess: nullptr = the reference's cold start; otherwise the interior start values (may be vh).
// zero_faces: zero boundary values even where the reference's rule would give Q/|r|.
JacobiResult hartree(dft_context* ctx, const Grid& g, const double* rho, double* vh, double tol, long max_sweeps,
                     const double* guess = nullptr, bool zero_faces = false);
// true when every face's last node lands exactly on the bound (the reference's boundary is then zero)
bool faces_exact(const Grid& g);
// The same solve on the library's fixed scratch array: no device allocation (grid_ops.cu).
// noalloc_scratch: the array's device address on `device` (must be current), looked up once.
double* noalloc_scratch(int device);
JacobiResult hartree_noalloc(dft_context* ctx, const Grid& g, const double* rho, double* vh, double tol,
                             long max_sweeps);

// Z-slab decomposition (zslab.cu).  A slab holds the global planes [z_lo, z_hi) of grid g.
// zslab_jacobi_init: the reference's face values (Q: total charge, used only on faces whose
// last node misses the bound) and a cold or `guess` interior.  zslab_jacobi_sweeps: `sweeps`
// Jacobi sweeps of the slab's interior planes (outermost planes fixed) from v_in (only read)
// into v_out (scratch: a third buffer of the slab's size), diffs[t] = max|dV| of sweep t over
// the owned planes [own_lo, own_hi) (global indices).  zslab_hamiltonian: H psi of the slab
// (owned planes exact with one halo plane per side).
void zslab_jacobi_init(dft_context* ctx, const Grid& g, int z_lo, int z_hi, double Q, const double* guess, double* v);
void zslab_jacobi_sweeps(dft_context* ctx, const Grid& g, int z_lo, int z_hi, int own_lo, int own_hi,
                         const double* rho, const double* v_in, double* v_out, double* scratch, int sweeps,
                         double* diffs);
void zslab_hamiltonian(dft_context* ctx, const Grid& g, int z_lo, int z_hi, const double* V, const double* psi,
                       double* hpsi, int nbands, long long ld);
// XC potentials of the slab (owned planes exact with two halo planes per side; va/vb may be
// NULL) and the owned planes' part of E_xc (returned; synchronises).
double zslab_xc(dft_context* ctx, const Grid& g, int z_lo, int z_hi, int own_lo, int own_hi, int kind,
                const double* na, const double* nb, double* va, double* vb);
// dV A^T B over the owned planes of a slab (the rank's part of the Gram product; ka x kb row-major)
void zslab_gram(dft_context* ctx, const Grid& g, int z_lo, int z_hi, int own_lo, int own_hi, const double* A,
                long long lda, int ka, const double* B, long long ldb, int kb, int precision, std::vector<double>& C);

// Monopole boundary option (grid_ops.cu): vc = Q erf(|r|/(sqrt 2 s))/|r| (Q = sum rho dV, returned)
// and rho_prime = rho + L_h vc / (4 pi) on the interior, so that V_H = V' + vc with V' the
// zero-face solution for rho_prime has the face values Q/|r|.  monopole_width: s for grid g.
double monopole_prepare(dft_context* ctx, const Grid& g, const double* rho, double* rho_prime, double* vc);
double monopole_width(const Grid& g);
// v = 0 on the six faces of g (the zero-face solvers' boundary)
void zero_faces(dft_context* ctx, const Grid& g, double* v);
// out = a + b (plain addition)
void add_into(dft_context* ctx, long long n, const double* a, const double* b, double* out);

// The context's device status word (allocated on first use) and its check: fails with
// DFT_CUDA_ERROR (and clears the word) when a kernel's bounded wait gave up since the last check.
int* device_status(dft_context* ctx);
void check_device_status(dft_context* ctx, const char* what);

// rho = a + b
void add2(dft_context* ctx, long long n, const double* a, const double* b, double* out);
// out = (a + b) + c
void add3(dft_context* ctx, long long n, const double* a, const double* b, const double* c, double* out);
// d = (1-m) d + m o   (mixDensity, MolecularSCFHelpers.cpp:27-44)
void mix(dft_context* ctx, long long n, double* d, const double* o, double m);

// out = max(0, sum_i c_i (a_i + beta r_i)) over m <= 16 history entries (Pulay mixing)
void pulay_combine(dft_context* ctx, long long n, int m, const double* const* a, const double* const* r,
                   const double* c, double beta, double* out);
// out = sum_i c_i a_i over m <= 16 fields (no clamp)
void combine(dft_context* ctx, long long n, int m, const double* const* a, const double* c, double* out);
// Kerker-screened density step for ns spin fields (ns = 1: closed shell, the field is n_alpha):
// x = (-lap_h + q2)^{-1} (r_0 + r_1) by two multigrid cycles (rtot: scratch for the sum), then
// a_s = max(0, a_s + beta (r_s - (q2/2) x)), i.e. the total-charge residual is multiplied by
// -lap/(-lap + q2) (the real-space Kerker factor G^2/(G^2 + q0^2)) and the spin residual is kept.
void kerker_update(dft_context* ctx, const Grid& g, int ns, double* const* a, const double* const* r, double* rtot,
                   double* x, double q2, double beta);
// out = a - b
void sub(dft_context* ctx, long long n, const double* a, const double* b, double* out);

// sum_p a[p]*b[p] (optionally * w[p]); deterministic block order
double dot(dft_context* ctx, long long n, const double* a, const double* b);
// sum_p a[p]*b[p]*c[p] evaluated as (a*b)*c per term
double dot3(dft_context* ctx, long long n, const double* a, const double* b, double c);

// relative L2 density difference (calculateMolecularDensityDifference)
double density_difference(dft_context* ctx, const Grid& g, const double* old_d, const double* new_d);

// XC potential (both spins) and/or energy.  va/vb may be null.  Returns E_xc if want_energy.
double xc(dft_context* ctx, const Grid& g, int kind, const double* na, const double* nb, double* va, double* vb,
          bool want_energy);
void xc_evaluate(dft_context* ctx, int kind, long long m, const double* na, const double* nb, const double* ga,
                 const double* gb, double* out5);

// density from a band block with host weights
void spin_density(dft_context* ctx, long long n, const double* psi, int nbands, long long ld, const double* occ_host,
                  double* out);
double kinetic_energy(dft_context* ctx, const Grid& g, const double* psi, int nbands, long long ld,
                      const double* occ_host);
// per-band <psi_b| -1/2 lap |psi_b> dV (face stencil), into out_host[nbands]
void kinetic_per_band(dft_context* ctx, const Grid& g, const double* psi, int nbands, long long ld, double* out_host);
void nuclear_potential(dft_context* ctx, const Grid& g, int nnuc, const int* Z, const double* xyz, double* vext);

// C (ka x kb, host) = dV A^T B: FP64 (davidson.cu) or on the tensor cores with a TF32 hi+lo
// split (gram_tc.cu).
// out = beta*out + alpha * in * Y (Y: k x m host row-major), FP64 (davidson.cu)
void rotate(dft_context* ctx, const Grid& g, const double* in, long long ldi, int k, const std::vector<double>& Y, int m,
            double* out, long long ldo, double alpha, double beta);
// X (m bands) = V (k bands) * Y (k x m, host row-major) on the tensor cores, TF32 hi+lo split
// (gram_tc.cu).
void rotate_tc(dft_context* ctx, const Grid& g, const double* V, long long ldv, int k, const std::vector<double>& Y,
               int m, double* X, long long ldx);
void gram_fp64(dft_context* ctx, const Grid& g, const double* A, long long lda, int ka, const double* B,
               long long ldb, int kb, std::vector<double>& C);
void gram_tc(dft_context* ctx, const Grid& g, const double* A, long long lda, int ka, const double* B, long long ldb,
             int kb, std::vector<double>& C);

// Block Davidson eigensolver (davidson.cu).
// One multigrid V(2,2) cycle from zero for (T + sigma_a) t_a = r_{src[a]} per band a (T the
// kinetic operator with psi = 0 outside the box), into T[a*ld ..] (precond_mg.cu), with
// sigma_a = max(-theta[src[a]], 1 Ha).  src_dev: device band indices into R and theta_dev.
void precondition_multigrid(dft_context* ctx, const Grid& g, const double* R, const int* src_dev, int nb,
                            const double* theta_dev, double* T, long long ld);

// `cycles` multigrid V(2,2) cycles (the first from zero, then iterative refinement) for
// (-lap_h + q2) x_a = src_a, x = 0 outside the box, for nb fields of ld points (precond_mg.cu):
// x ~ (-lap_h + q2)^{-1} src, a fixed linear map.
void screened_poisson_vcycle(dft_context* ctx, const Grid& g, const double* src, int nb, double q2, double* x,
                             long long ld, int cycles = 1);

// X_a ~ (T + sigma_a)^-1 R_a for nb fields by `cycles` multigrid cycles with iterative refinement
// (the first from zero), sigma on the device; res and e: scratch of nb x ld doubles each.
void helmholtz_refine(dft_context* ctx, const Grid& g, const double* R, int nb, const double* sigma_dev, double* X,
                      long long ld, int cycles, double* res, double* e);

struct EigOpts {
    double tol = 1e-7;
    int max_iterations = 2000;
    int max_subspace = 3;
    int verbose = 0;
    int precond_steps = 4;  // 0 = the reference's diagonal preconditioner; -3 = learned (precond_net)
    dft_pnet* precond_net = nullptr;
    // training-data hook: called every iteration with the residual block and its active bands
    void (*harvest)(void* user, const double* R, long long ld, const int* active, int na, const double* theta) =
        nullptr;
    void* harvest_user = nullptr;
    int mixed_precision = 0;       // 1 = tensor-core (TF32 hi+lo) Gram products while residuals are large
    double mixed_switch = 1e-3;    // occupied residual below which the solver switches to FP64
};
// start/nstart: an optional start basis of nstart vectors (leading dimension ld) that replaces
// psi's contents and the seeds; the first Rayleigh-Ritz step takes the lowest nbands from it.
int solve_orbitals(dft_context* ctx, const Grid& g, const double* V, int nocc, int nbands, double* psi,
                   long long ld, bool init, double* eig_host, double* resid_host, const EigOpts& o,
                   const double* start = nullptr, int nstart = 0);

// Launch-shape autotuner (autotune.cu): sets the context's H psi and Jacobi knobs for (g, nbands).
void autotune(dft_context* ctx, const Grid& g, int nbands, dft_autotune_report* rep);

// Molecular SCF (scf.cu).
void scf_molecule(dft_context* ctx, const dft_grid* grid, int nnuc, const int* Z, const double* xyz, int charge,
                  int multiplicity, int kind, const dft_scf_opts* opts, dft_scf_result* res);

// Radial atoms, one persistent launch (radial.cu).
void solve_atoms(dft_context* ctx, int nruns, const int* Z, const int* kinds, long points, double rmax,
                 dft_atom_result* results);
// The same batch for nz atoms with one functional, keeping the converged atoms on the device:
// dens (nz x points) the total density n(r), orbs (nz x RADIAL_MAX_SHELLS x points) the radial
// functions u_nl(r) = r R_nl(r) of the alpha shells, listed per atom as (n, l) in shells.
constexpr int RADIAL_MAX_SHELLS = 8;
void radial_atom_tables(dft_context* ctx, int nz, const int* Z, int kind, long points, double rmax, double* dens,
                        double* orbs, std::vector<std::vector<std::array<int, 2>>>& shells);

// Number of start vectors atomic_start writes: 2l + 1 per occupied (n, l) shell of every atom.
int atomic_orbital_count(int nnuc, const int* Z);
// Superposition start of the molecular SCF (atomic_start.cu): the radial atoms of every nucleus'
// element (functional `kind`, 2000 points, r_max 30 bohr) are solved in one batch; their total
// densities, summed at every node and scaled to ne_a + ne_b electrons, split in the ratio
// ne_a : ne_b, give da and db.  When basis != nullptr it also receives one start vector per
// occupied atomic orbital (u_nl(r)/r times 1, x/r, y/r or z/r), at most max_basis of them,
// band-major with leading dimension ld; returns the number written.
int atomic_start(dft_context* ctx, const Grid& g, int nnuc, const int* Z, const double* xyz, int kind, int ne_a,
                 int ne_b, double* da, double* db, double* basis, long long ld, int max_basis);

}  // namespace dftb
