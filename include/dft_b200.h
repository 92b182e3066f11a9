/*
 * dft_b200 — C ABI of the B200-native real-space Kohn–Sham engine.
 *
 * This is the drop-in boundary for the reference's (willandru/DFT) C++ driver API:
 * every entry point below replaces one reference function, cited beside it, and a
 * header-only C++ shim (dft_b200.hpp) re-exports the reference signatures on top.
 * Plain C types only: no CUDA, torch or STL types cross this boundary.
 *
 * Conventions
 *  - Status: every function returns dft_status_t; on failure dft_last_error_message()
 *    holds a one-line reason (thread-local).  The reference's exceptions map to
 *    DFT_INVALID_ARGUMENT (std::invalid_argument) and DFT_NOT_CONVERGED / DFT_SINGULAR
 *    (std::runtime_error).
 *  - Memory: entry points ending in _dev take DEVICE pointers (from dft_device_alloc or
 *    any cudaMalloc'd buffer on the context's device) and run stream-ordered on the
 *    context's stream; results are ready after dft_context_synchronize().  Entry points
 *    without the suffix take HOST pointers and block until done.
 *  - Grids: point (i,j,k) lives at (k*ny + j)*nx + i, x fastest; spacing
 *    (max-min)/(n-1) exactly as CartesianGrid (reference CartesianGrid.cpp:5-48).
 *    A band block is band-major: band b starts at psi + b*ld (ld >= nx*ny*nz).
 *  - Units: Hartree atomic units.  One context = one GPU; calls on one context are not
 *    thread-safe.
 */
#ifndef DFT_B200_H
#define DFT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    DFT_OK = 0,
    DFT_INVALID_ARGUMENT = 1, /* reference: std::invalid_argument */
    DFT_NOT_CONVERGED = 2,    /* reference: std::runtime_error from the Davidson solver */
    DFT_CAP_REACHED = 3,      /* an iteration cap was hit where the reference would throw */
    DFT_SINGULAR = 4,         /* reference: singular tridiagonal pivot / nucleus on a node */
    DFT_CUDA_ERROR = 5,       /* a CUDA runtime call failed */
    DFT_NUMERICAL = 6         /* NaN/Inf detected in device data */
} dft_status_t;

typedef enum { DFT_XC_PZ81 = 0, DFT_XC_PBE96 = 1 } dft_xc_kind; /* PZ81.h / PBE96.h */

/* CartesianGrid(nx,ny,nz,xmin,xmax,ymin,ymax,zmin,zmax), reference CartesianGrid.h:5-60 */
typedef struct {
    long nx, ny, nz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
} dft_grid;

typedef struct dft_context dft_context;
typedef struct dft_pnet dft_pnet; /* learned Poisson start network (see the end of this header) */

const char* dft_last_error_message(void);
const char* dft_version(void);

/* ---- context and device memory (no reference counterpart: the reference has no device) ---- */
dft_status_t dft_context_create(int device, dft_context** out);
dft_status_t dft_context_destroy(dft_context* ctx);
/* Waits for the context's stream.  Also fails with DFT_CUDA_ERROR when a kernel launched since
 * the last call gave up a bounded wait (the TMA H psi ring, "hpsi_variant" = 2); the context
 * stays usable. */
dft_status_t dft_context_synchronize(dft_context* ctx);
/* Kernel-shape knobs.  Keys:
 *   "jacobi_sweeps_per_launch": 0 = auto (default), -2 = the whole solve in the shared memory
 *                               of one 16-block cluster (small grids), -1 = the whole solve in
 *                               one persistent (cooperative) launch, 1 = one sweep per launch,
 *                               2, 4 or 8 = temporally blocked sweeps per launch (results are
 *                               identical for every value).
 *   "network_tensor_cores":     1 (default) = the Poisson-start network's 16- and 32-channel
 *                               convolutions on tcgen05, 0 = FP32 CUDA cores (results agree to
 *                               BF16 rounding, not bit for bit).
 *   "hpsi_bands_per_thread":    0 = auto (default), 1, 2 or 4 bands marched together by each
 *                               thread of the H psi kernel (8 counts as 4), or with
 *                               "hpsi_variant" = 2 the bands (1, 2, 4, 8) each block walks
 *                               (results identical for every value).
 *   "multigrid_graphs":         1 (default) = each Poisson multigrid cycle is captured once per
 *                               grid and buffers as a CUDA graph and replayed; 0 = launched kernel
 *                               by kernel (same results).
 *   "tensor_core_ring":         0 (default) = the tensor-core Gram product stages its FP64 slices
 *                               through registers; 1 = through a 2-deep cp.async shared-memory
 *                               ring (even leading dimensions, 16-byte-aligned blocks, <= 128
 *                               columns per tile; otherwise the register path).  Same results.
 *   "tensor_core_tma":          0 (default) = as "tensor_core_ring" says; 1 = the tensor-core Gram
 *                               product loads 16-point FP64 slices with TMA (cp.async.bulk.tensor,
 *                               128-byte swizzle) into a 4-stage mbarrier ring (2 stages for
 *                               256-column tiles) and splits them from shared memory (even
 *                               leading dimensions, 16-byte-aligned blocks; otherwise the other
 *                               paths).  Same accuracy class (TF32 hi+lo, FP32 accumulation).
 *   "hpsi_variant":             0 (default) = the H psi kernel reads x/y neighbours through L1;
 *                               1 = through a shared-memory plane tile (at most 2 bands per
 *                               thread); 2 = plane tiles with their halo loaded by TMA
 *                               (cp.async.bulk.tensor) into a 6-stage shared-memory ring, each
 *                               block walking hpsi_bands_per_thread bands (0 = 4) of its column
 *                               tile; needs nx and ld even and a 16-byte-aligned psi, else 0 is
 *                               used; 3 = the single-band march of 0 with the next plane's loads
 *                               issued one step ahead.  Results identical for every value.
 *   "grid_barrier_poll_limit":  0 = 2^24 (default): polls a block of the persistent Jacobi
 *                               launch makes at a grid barrier before it gives up; the solve then
 *                               fails with DFT_CUDA_ERROR and the context stays usable.
 *   "hpsi_zchunk":              0 = auto (default), else the number of z-planes each block of the
 *                               register-march H psi kernels walks (same results for every value).
 *   "multigrid_fused_restriction": 1 (default) = the Poisson multigrid restricts in one 3-D pass
 *                               on fine grids up to 64^3 (0: three separable passes).
 *   "multigrid_coarsest_sor":   1 (default) = the coarsest multigrid level is solved by red-black
 *                               SOR at the optimal relaxation (0: 8 Jacobi sweeps per point of the
 *                               longest axis).
 *   "orthonormalise_adaptive":  1 (default) = the FP64 orthonormalisation of new eigensolver
 *                               directions stops after one projected Cholesky QR pass when its
 *                               estimated loss of orthogonality (eps * cancellation * condition
 *                               bound) is below 1e-12; 0 = always two passes.
 *   "radial_pivot_exponent":    -14 (default): a pivot of the radial inverse iteration's Thomas
 *                               factorisation below 10^value in magnitude is singular; the run's
 *                               status becomes DFT_SINGULAR (reference NumericalMethods.cpp:105-122). */
dft_status_t dft_context_set_tuning(dft_context* ctx, const char* key, long value);

/* Autotuner (no reference counterpart): times every bit-identical launch variant of the H psi
 * kernel (1, 2, 4 bands per thread, on min(nbands, 16) bands, and the TMA plane ring with 1, 2,
 * 4, 8 bands per block where the grid allows it) and of the Jacobi Poisson solve
 * (sweeps per launch -2, -1, 1, 2, 4, 8; 64 sweeps) on grid g with CUDA events on the context's
 * stream and remembers the fastest of each for grid g in the context: kernels on g use it
 * wherever the "hpsi_bands_per_thread" or "jacobi_sweeps_per_launch" knob is 0 (auto) (the H psi
 * kernel variant too, while "hpsi_variant" is 0), and a
 * second call for g times nothing.  report may be NULL; a time of -1 marks a variant that does
 * not apply (e.g. a grid too large for the cluster-resident Jacobi).  Allocates
 * (2 min(nbands,16) + 3) x N doubles while it runs. */
typedef struct {
    int hpsi_bands_per_thread;     /* chosen */
    double hpsi_ms[3];             /* 1, 2, 4 bands per thread */
    int jacobi_sweeps_per_launch;  /* chosen */
    double jacobi_us_per_sweep[6]; /* -2, -1, 1, 2, 4, 8 */
    int cached;                    /* 1: the choice was remembered, nothing was timed */
    int hpsi_variant;              /* chosen: 0 = the register march (hpsi_ms), 2 = the TMA ring,
                                      3 = the prefetching single-band march */
    double hpsi_tma_ms[4];         /* TMA plane ring with 1, 2, 4, 8 bands per block (-1: not eligible) */
    double hpsi_prefetch_ms;       /* the prefetching single-band march */
    int hpsi_zchunk;               /* chosen z-march length per block of the register march (0 = auto) */
    double hpsi_zchunk_ms[5];      /* the chosen register march with 16, 32, 64, 96, 192 planes per block */
} dft_autotune_report;
dft_status_t dft_autotune(dft_context* ctx, const dft_grid* g, int nbands, dft_autotune_report* report);
/* The cudaStream_t the context launches on, as an opaque handle (for event timing). */
void* dft_context_stream(dft_context* ctx);
/* Number of kernels this context has launched so far (diagnostics, bench accounting). */
long long dft_context_launch_count(dft_context* ctx);
/* Named counters of this context (diagnostics): "launches" (as above), "tensor_core_products"
 * (tcgen05 Gram products and subspace rotations of the eigensolver); -1 for an unknown name. */
long long dft_context_counter(dft_context* ctx, const char* name);
dft_status_t dft_device_alloc(dft_context* ctx, size_t bytes, void** out);
dft_status_t dft_device_free(dft_context* ctx, void* ptr);
dft_status_t dft_copy_h2d(dft_context* ctx, void* dst, const void* src, size_t bytes);
dft_status_t dft_copy_d2h(dft_context* ctx, void* dst, const void* src, size_t bytes);

/* ---- 3D operators on device buffers ---------------------------------------------------- */

/* applyMolecularKohnShamHamiltonian (reference KohnShamHamiltonianMolecule.h:7-11,
 * KohnShamHamiltonianMolecule.cpp:7-183) over a block of nbands bands:
 * hpsi_b = -1/2 lap_h psi_b + V psi_b, psi = 0 outside the box.  Bit-identical to the
 * reference for each band. */
dft_status_t dft_apply_hamiltonian_dev(dft_context* ctx, const dft_grid* g, const double* V, const double* psi,
                                       double* hpsi, int nbands, long ld);

/* calculateHartreePotential (reference HartreePotentialMolecule.h:7-10,
 * HartreePotentialMolecule.cpp:99-324): boundary fill Q/|r| (zero on a face), then Jacobi
 * sweeps for lap V = -4 pi rho from a cold (zero) interior start, stopping at the first
 * sweep whose max|dV| < tol or after max_sweeps sweeps (tol = 1e-8, max_sweeps = 10000
 * reproduce the reference bit-for-bit).  sweeps_out (host, may be NULL) receives the
 * number of sweeps run; last_diff_out (host, may be NULL) the last sweep's max|dV|. */
dft_status_t dft_hartree_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh, double tol,
                             long max_sweeps, long* sweeps_out, double* last_diff_out);

/* The Hartree solve of dft_hartree_dev (same arguments, same bit-identical results) for
 * callers that cannot let a library allocate device memory: applications whose own pooled
 * allocator owns the device memory budget, or plugins running inside such an
 * application's compute step, where cudaMalloc/cudaFree would also stall the device.
 * This entry point calls no cudaMalloc, cudaFree or other allocating routine; its scratch
 * (the second Jacobi iterate and the control words) is a fixed array compiled into the
 * library, so every GPU on which a context is created holds 16 MiB + 128 B until the
 * process exits.  dft_context_create looks up the array's device address, which also
 * makes CUDA load it where modules load lazily, so this entry point neither loads nor
 * allocates anything.  Limit: nx*ny*nz <= 2,097,152 points (128^3); larger grids are
 * rejected with DFT_INVALID_ARGUMENT.  Every call runs one Jacobi sweep per launch,
 * whatever the "jacobi_sweeps_per_launch" tuning key says, so small grids take more
 * launches than with dft_hartree_dev.  All calls share the array: calls that overlap on
 * the GPU (several streams or contexts on one device at once) race on it.  No counterpart
 * in the reference. */
dft_status_t dft_hartree_noalloc_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh, double tol,
                                     long max_sweeps, long* sweeps_out, double* last_diff_out);

/* Hartree potential with V = Q/|r| on every face (Q = sum rho dV, |r| from the origin), the
 * boundary of dft_scf_opts.hartree_boundary = 1: a Gaussian compensation charge of width
 * (smallest origin-face distance)/8 carries Q, the remainder is solved by the Jacobi sweeps of
 * dft_hartree_dev with zero faces (same tol / max_sweeps stop rule) and the compensation's
 * potential is added back.  The origin must lie more than four spacings inside every face
 * (DFT_INVALID_ARGUMENT otherwise).  Allocates two N-point scratch arrays per call.  No
 * counterpart in the reference, whose faces follow dft_hartree_dev. */
dft_status_t dft_hartree_monopole_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh, double tol,
                                      long max_sweeps, long* sweeps_out, double* last_diff_out);

/* ---- z-slab decomposition (one rank's slab; the halo exchange and the reductions over ranks
 * are the caller's) ---------------------------------------------------------------------
 * A slab is the global planes [z_lo, z_hi) of grid g (x fastest, (k - z_lo)*nx*ny + j*nx + i),
 * holding the rank's own planes plus halo planes copied from its neighbours.  The reference
 * has no decomposition; these split its functions over ranks with bit-identical results. */

/* Initial state of the Jacobi solve of dft_hartree_dev on a slab (reference
 * HartreePotentialMolecule.cpp:37-95, :152-155): the reference's face values where the slab
 * meets a face of g, Q/|r| with Q the total charge (used only on faces whose last node misses
 * the bound; 0 on every grid whose nodes land on the bounds), interior 0, or the interior of
 * guess (device, same slab layout) when guess is not NULL.  v: device, nx*ny*(z_hi - z_lo).
 * Synchronises. */
dft_status_t dft_zslab_jacobi_init_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, double Q,
                                       const double* guess, double* v);

/* `sweeps` Jacobi sweeps of dft_hartree_dev's loop (reference HartreePotentialMolecule.cpp:
 * 207-321) on a slab, from v_in into v_out: every plane of the slab except its first and last
 * is updated, so with T halo planes per side the rank's own planes are exact for up to T
 * sweeps.  v_in is only read, so a block of sweeps that passed the stop can be rerun from it.
 * diffs (device, `sweeps` doubles): max|dV| of each sweep over the owned planes
 * [own_lo, own_hi) (global indices; every owned plane that g's interior contains must be an
 * inner plane of the slab).  The maximum of diffs[t] over ranks is the single-domain loop's
 * max|dV| of that sweep.  rho, v_in, v_out, scratch: distinct device buffers of the slab's
 * size.  Synchronises. */
dft_status_t dft_zslab_jacobi_sweeps_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, int own_lo,
                                         int own_hi, const double* rho, const double* v_in, double* v_out,
                                         double* scratch, int sweeps, double* diffs);

/* dft_apply_hamiltonian_dev on a slab (reference KohnShamHamiltonianMolecule.cpp:78-177):
 * with one halo plane per side (none at the faces of g) the owned planes of hpsi are
 * bit-identical to the whole-grid result.  ld >= nx*ny*(z_hi - z_lo). */
dft_status_t dft_zslab_hamiltonian_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, const double* V,
                                       const double* psi, double* hpsi, int nbands, long ld);

/* dft_xc_dev on a slab (reference ExchangeCorrelationMolecule.cpp:576-842): va/vb (device, the
 * slab's size, either may be NULL) get the XC potentials, bit-identical to the whole-grid
 * result on the owned planes [own_lo, own_hi) when the slab holds two planes beyond them on
 * each side (or ends at a face of g; DFT_INVALID_ARGUMENT otherwise).  exc_out (host, may be
 * NULL): the owned planes' part of E_xc; the ranks' parts add up to E_xc (summed in a different
 * order than the whole grid's).  Synchronises. */
dft_status_t dft_zslab_xc_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, int own_lo, int own_hi,
                              dft_xc_kind kind, const double* na, const double* nb, double* va, double* vb,
                              double* exc_out);

/* The owned planes' part of dft_gram_dev's product: dV * A^T B summed over the points of the
 * planes [own_lo, own_hi) of a slab (A: ka bands, B: kb bands, leading dimensions >= the slab's
 * size), into C_host (ka x kb, row-major).  The ranks' parts add up to the whole grid's
 * product. */
dft_status_t dft_zslab_gram_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, int own_lo, int own_hi,
                                const double* A, long lda, int ka, const double* B, long ldb, int kb, int precision,
                                double* C_host);

/* calculateHartreeEnergy (reference HartreePotentialMolecule.cpp:326-379): 1/2 sum rho V dV. */
dft_status_t dft_hartree_energy_dev(dft_context* ctx, const dft_grid* g, const double* rho, const double* vh,
                                    double* energy_out);

/* calculateMolecularSpinExchangeCorrelationPotential for spin 0 and 1 in one pass, plus
 * calculateMolecularExchangeCorrelationEnergy (reference ExchangeCorrelationMolecule.h:8-21,
 * ExchangeCorrelationMolecule.cpp:576-842).  va/vb may be NULL to skip a spin; exc_out
 * (host, may be NULL) receives E_xc. */
dft_status_t dft_xc_dev(dft_context* ctx, const dft_grid* g, dft_xc_kind kind, const double* na, const double* nb,
                        double* va, double* vb, double* exc_out);

/* XCFunctional::evaluate (reference XCFunctional.h:15-22) at m independent points;
 * out5 is m x {energyPerElectron, potentialAlpha, potentialBeta, gradCoefAlpha, gradCoefBeta}. */
dft_status_t dft_xc_evaluate_dev(dft_context* ctx, dft_xc_kind kind, long m, const double* na, const double* nb,
                                 const double* ga, const double* gb, double* out5);

/* calculateMolecularSpinDensity (reference ElectronDensityMolecule.cpp:5-76):
 * out = sum_b occ[b] psi_b^2 in band order; occ is a host array of nbands weights. */
dft_status_t dft_spin_density_dev(dft_context* ctx, long npoints, const double* psi, int nbands, long ld,
                                  const double* occ, double* out);

/* calculateMolecularKineticEnergy (reference TotalEnergyMolecule.cpp:13-199, the face
 * stencil of existing neighbours): sum_b occ[b] <psi_b| -1/2 lap |psi_b> dV. */
dft_status_t dft_kinetic_energy_dev(dft_context* ctx, const dft_grid* g, const double* psi, int nbands, long ld,
                                    const double* occ, double* energy_out);

/* NuclearPotential::calculate (reference NuclearPotential.cpp:6-76); Z and xyz are HOST
 * arrays of nnuc charges and positions.  DFT_SINGULAR if a node coincides with a nucleus. */
dft_status_t dft_nuclear_potential_dev(dft_context* ctx, const dft_grid* g, int nnuc, const int* Z,
                                       const double* xyz, double* vext);

/* ---- eigensolver --------------------------------------------------------------------- */

typedef struct {
    double tol;          /* residual norm (dV-weighted) for occupied bands; 1e-7 (reference :19) */
    int max_iterations;  /* block iterations cap */
    int max_subspace;    /* basis size cap in multiples of nbands (>= 2) */
    int verbose;         /* 1: per-iteration lines on stderr */
    int preconditioner;  /* 0: the reference's diagonal (theta - diag)^-1 (EigenvalueSolverMolecule.cpp:521-555);
                            k > 0: k damped-Jacobi smoothing steps on (T + sigma) t = r (default 4);
                            -1: one multigrid V(2,2) cycle on (T + sigma) t = r, all bands batched;
                            -2: -1 on grids of 32^3 points or more, 4 below;
                            -3: -1 plus the learned correction of preconditioner_net, trained by
                                dft_pnet_train_preconditioner */
    int mixed_precision; /* 1: Gram products on the tensor cores (TF32 hi+lo split, FP32 accumulation)
                            until the occupied residuals fall below 1e-3, then FP64 to the end */
    dft_pnet* preconditioner_net; /* the network of preconditioner -3 (not owned), else NULL */
} dft_eig_opts;

/* X (m x N, leading dimension ldx, device) = V (k x N, ldv, device) * Y (k x m, host,
 * row-major).  precision 0 = FP64, 1 = tensor cores (TF32 hi+lo split).  The block
 * eigensolver's subspace rotation, exposed for testing; no counterpart in the reference (its
 * combinations are EigenvalueSolverMolecule.cpp:451-481). */
dft_status_t dft_rotate_dev(dft_context* ctx, const dft_grid* g, const double* V, long ldv, int k, const double* Y,
                            int m, double* X, long ldx, int precision);

/* x ~ (-lap_h + q2)^{-1} src by `cycles` multigrid V(2,2) cycles, the first from zero and the
 * rest refining (7-point Laplacian, x = 0 outside the box; src, x: device, N doubles; q2 > 0).
 * The screening solve of the Kerker mixer (dft_scf_opts.kerker_q0, which uses 2 cycles),
 * exposed for testing; no counterpart in the reference, whose mixer is linear
 * (MolecularSCFHelpers.cpp:27-44). */
dft_status_t dft_screened_poisson_dev(dft_context* ctx, const dft_grid* g, const double* src, double* x, double q2,
                                      int cycles);

/* dV * A^T B for band blocks A (ka x N, leading dimension lda) and B (kb x N), result in
 * C_host (ka x kb, row-major).  precision 0 = FP64, 1 = tensor cores (TF32 hi+lo split).
 * The block eigensolver's Gram product, exposed for testing; no counterpart in the reference
 * (its dot products are EigenvalueSolverMolecule.cpp:35-47). */
dft_status_t dft_gram_dev(dft_context* ctx, const dft_grid* g, const double* A, long lda, int ka, const double* B,
                          long ldb, int kb, int precision, double* C_host);

/* solveMolecularOrbitals (reference EigenvalueSolverMolecule.h:20-28,
 * EigenvalueSolverMolecule.cpp:1233-1300): the lowest nocc eigenpairs of H = -1/2 lap_h + V,
 * computed by a block Davidson method over nbands >= nocc bands.  psi (nbands x ld, device)
 * holds the start vectors on entry (any non-zero block; orthonormalised internally) and the
 * dV-normalised eigenvectors on exit; eig (host, nbands) the eigenvalues.  When init is 0,
 * psi's contents are ignored and the reference's Gaussian x polynomial seeds are used.
 * iterations_out (host, may be NULL).  DFT_NOT_CONVERGED if the occupied residuals stay
 * above tol after max_iterations (reference: runtime_error). */
dft_status_t dft_solve_orbitals_dev(dft_context* ctx, const dft_grid* g, const double* V, int nocc, int nbands,
                                    double* psi, long ld, int init, double* eig, const dft_eig_opts* opts,
                                    int* iterations_out);

/* ---- SCF drivers (host in, host out) ------------------------------------------------- */

typedef enum {
    DFT_POISSON_COLD = 0,     /* zero interior, as HartreePotentialMolecule.cpp:152-155 */
    DFT_POISSON_PREVIOUS = 1, /* the previous SCF iteration's potential for the same density slot */
    DFT_POISSON_NETWORK = 2,  /* coarse-grid solve plus the network's correction (dft_poisson_start_dev) */
    DFT_POISSON_COARSE = 3,   /* coarse-grid solve alone */
    DFT_POISSON_HYBRID = 4,   /* DFT_POISSON_NETWORK (coarse alone when poisson_net is NULL) for the
                                 first solve of each density slot, DFT_POISSON_PREVIOUS afterwards */
    DFT_POISSON_MULTIGRID = 5 /* multigrid cycles from the previous potential (first solve: from the
                                 coarse or network start), then Jacobi with the unchanged stop rule */
} dft_poisson_start;

typedef struct {
    int max_iterations;      /* 250 (DFTConstants.h:13) */
    double energy_tol;       /* 1e-11 (DFTConstants.h:16) */
    double density_tol;      /* 1e-9  (DFTConstants.h:15) */
    double ks_tol;           /* 1e-7  (DFTConstants.h:17) */
    double stop_abs_de;      /* > 0: also stop as soon as |dE| < stop_abs_de (time-to-|dE| metric) */
    double poisson_tol;      /* 1e-8  (HartreePotentialMolecule.cpp:15) */
    long poisson_max_sweeps; /* 10000 (HartreePotentialMolecule.cpp:14) */
    int extra_bands;         /* unoccupied buffer bands per spin in the block eigensolver */
    dft_eig_opts eig;        /* eigensolver options (tol = 1e-7 reproduces the reference) */
    int verbose;             /* 1: one line per SCF iteration on stderr */
    /* Start of each Poisson solve (no counterpart in the reference, which always starts
     * from zero): DFT_POISSON_COLD reproduces the reference. */
    int poisson_start;       /* dft_poisson_start */
    dft_pnet* poisson_net;   /* network for DFT_POISSON_NETWORK (not owned) */
    /* Density mixing and eigensolver tolerance (no counterpart in the reference; the defaults
     * 0 keep its linear mixer, SelfConsistentFieldMolecule.cpp:447-484, and its fixed tolerance). */
    int mixer;               /* 0: linear with the adaptive factor; 1: Pulay (DIIS) on n_out - n_in */
    int pulay_depth;         /* history length for the Pulay mixer (0 = 16, at most 16) */
    double pulay_beta;       /* step along the extrapolated residual (0 = 0.5) */
    int adaptive_eig_tol;    /* 1: eigensolver tolerance max(eig.tol, min(1e-3, 0.1 * previous dRho)) */
    double smearing_kt;      /* > 0: Fermi-Dirac occupations at this temperature (Ha) over the extra
                                bands instead of the reference's integer aufbau (0) */
    double kerker_q0;        /* > 0: Kerker screening of the total-charge residual in either mixer,
                                -lap/(-lap + q0^2) by one multigrid cycle (bohr^-1; 0 = off) */
    double stop_abs_deig;    /* > 0: the stop_abs_de stop also needs every occupied eigenvalue to have
                                changed by less than this since the previous iteration (the energy is
                                second order in the density error, eigenvalues first order) */
    const char* log_path;    /* non-NULL: one JSON object per SCF iteration (the dft_scf_iteration
                                fields, energy components, the levels around the Fermi level per
                                spin) and a final {"result": ...} line, written to this file; the
                                reference prints the same quantities as tables
                                (MolecularSCFHelpers.cpp:251-513) */
    int autotune;            /* 1: run dft_autotune for the grid and band count first (launch shapes
                                only; results are bit-identical) */
    int initial_density;     /* 0: orbitals of the bare nuclear potential, as the reference
                                (buildInitialMolecularDensities, MolecularSCFHelpers.cpp:515-579);
                                1: superposed radial atoms of the same functional (batched radial
                                SCF, SelfConsistentField.cpp:539-786), scaled to the electron count,
                                and their occupied atomic orbitals as the first eigensolve's start */
    int hartree_boundary;    /* 0: the reference's face values (Q/|r| only on a face whose last node
                                misses the bound by rounding, else 0; HartreePotentialMolecule.cpp:45-94);
                                1: Q/|r| on every face (monopole), through a Gaussian compensation
                                charge and the same zero-face solvers; the wall states that zero
                                faces bind for many electrons do not form */
    int poisson_predict;     /* 1: start each V_H(n_in) solve (any poisson_start but COLD) from the
                                mixer's own combination of the stored V_H(n_in,i) and V_H(n_out,i)
                                (V_H is linear in n), instead of the slot's previous potential (0);
                                2: as 1, and each V_H(n_out) solve from V_H(n_in) plus the previous
                                iteration's V_H(n_out) - V_H(n_in).  The stop rule is unchanged;
                                only the cycles/sweeps to reach it drop */
    int poisson_fixed_point; /* 1: with DFT_POISSON_MULTIGRID the cycles of every solve go on until the
                                next Jacobi update is below tol (1 - rho_Jacobi) / 2, so each V_H is
                                at the Jacobi fixed point to ~tol instead of tol / (1 - rho) (the
                                eigenvalues are first order in that error); the Jacobi stop rule
                                that follows is unchanged.  0 (default): cycles to tol / 2 */
    double stop_abs_drho;    /* > 0: the stop_abs_de stop also needs the density difference below this.
                                The reported energy is first order in n_out - n_in: on H2O 64^3 a Pulay
                                plateau at dRho ~7e-7 kept |dE| and the eigenvalue changes below 1e-7
                                while E_tot was 1.2e-6 Ha from the fixed point */
} dft_scf_opts;

/* Per-iteration record: the reference's iteration table (MolecularSCFHelpers.cpp:264-352)
 * plus device phase times that the reference leaves at zero. */
typedef struct {
    int iteration;
    double energy, energy_difference, density_difference, ks_residual, mixing;
    long poisson_sweeps_in, poisson_sweeps_out;
    int eig_iterations_alpha, eig_iterations_beta;
    double ms_hartree, ms_xc, ms_orbitals, ms_density, ms_energy, ms_total;
    double eigenvalue_difference;  /* max |change| of the occupied eigenvalues since the previous iteration */
    int poisson_cycles_in, poisson_cycles_out;  /* multigrid cycles before the Jacobi stop rule
                                                   (DFT_POISSON_MULTIGRID start; 0 otherwise) */
} dft_scf_iteration;

typedef struct {
    /* EnergyComponents (reference DFTData.h:47-54) */
    double kinetic, external, hartree, exchange_correlation, nuclear_repulsion, total;
    int iterations, converged;
    double density_difference, energy_difference, max_ks_residual;
    int n_alpha, n_beta;
    double* eigenvalues;            /* caller buffer, >= n_alpha + n_beta entries (alpha then beta), or NULL */
    double* alpha_density;          /* caller buffers of N doubles, or NULL */
    double* beta_density;
    double* alpha_potential;        /* effective potentials of the last iteration (N doubles each), or NULL */
    double* beta_potential;
    double* orbitals;               /* caller buffer of (n_alpha + n_beta) x N doubles (alpha then beta), or NULL */
    dft_scf_iteration* history;     /* caller buffer of history_capacity records, or NULL */
    int history_capacity, history_len;
    double seconds;                 /* wall time of the solve */
    /* MolecularSCFConvergenceAnalysis (reference MolecularSCFHelpers.h:47-72): the last
     * iteration meeting each of the three stop criteria (0 = none) and the smallest value each
     * measure reached; the final values are energy_difference, density_difference and
     * max_ks_residual above */
    int last_energy_criterion_iteration, last_density_criterion_iteration, last_ks_criterion_iteration;
    double min_energy_difference, min_density_difference, min_ks_residual, final_mixing;
} dft_scf_result;

void dft_scf_default_options(dft_scf_opts* opts);

/* solveMolecularSelfConsistentField (reference SelfConsistentFieldMolecule.h:8-14,
 * SelfConsistentFieldMolecule.cpp:50-561; iteration MolecularSCFIteration.cpp:12-252):
 * nuclei Z[nnuc] at xyz[3*nnuc] (host), charge, multiplicity (1 = closed shell, beta := alpha),
 * functional kind.  Fills *result (host).  Returns DFT_OK whether or not the SCF converged
 * (result->converged says which), as the reference does. */
dft_status_t dft_scf_molecule(dft_context* ctx, const dft_grid* g, int nnuc, const int* Z, const double* xyz,
                              int charge, int multiplicity, dft_xc_kind kind, const dft_scf_opts* opts,
                              dft_scf_result* result);

/* ---- radial atoms --------------------------------------------------------------------- */

typedef struct {
    int Z;
    int kind;                      /* dft_xc_kind */
    double kinetic, external, hartree, exchange_correlation, total; /* EnergyComponents */
    int iterations, converged;
    double density_difference, max_ks_residual;
    int n_orbitals;                /* occupied (n,l,spin) orbitals, alpha then beta */
    double eigenvalues[16];
    int status;                    /* dft_status_t of this run */
} dft_atom_result;

/* solveAtom / solveSelfConsistentField (reference AtomicDFT.h:7-11, AtomicDFT.cpp:7-42,
 * SelfConsistentField.cpp:539-786) for nruns independent atoms (Z[r] in 1..30 with the
 * reference's configurations, kinds[r]) on RadialGrid(points, rmax), all advanced by one
 * persistent kernel launch, one thread block per run.  results: host array of nruns. */
dft_status_t dft_solve_atoms(dft_context* ctx, int nruns, const int* Z, const int* kinds, long points, double rmax,
                             dft_atom_result* results);

/* ---- learned Poisson start (no counterpart in the reference) ------------------------- */
/* A coarse grid with the same bounds and about a quarter of the points per axis carries the
 * long-range part of V_H: the density is restricted to it with the transposed trilinear
 * weights (charge-conserving), solved there by the same Jacobi kernels and interpolated back.
 * A 3-level convolutional network (BF16 activations, FP32 accumulation, about 1.5e5
 * parameters) predicts the remaining short-range correction from the density and the
 * interpolated coarse potential.  Jacobi then runs from that start with the unchanged stop
 * rule.  Parameters are FP32 on the host side of these calls. */

dft_status_t dft_pnet_create(dft_context* ctx, int in_channels, unsigned long long seed, dft_pnet** out);
dft_status_t dft_pnet_destroy(dft_pnet* net);
dft_status_t dft_pnet_num_params(const dft_pnet* net, size_t* n);
dft_status_t dft_pnet_get_params(dft_context* ctx, dft_pnet* net, float* host, size_t n);
dft_status_t dft_pnet_set_params(dft_context* ctx, dft_pnet* net, const float* host, size_t n);

/* One forward and backward pass on an (nx, ny, nz) volume: input x[N][in_channels] and
 * target t[N] (host, x fastest), loss = mean over interior points of (y - t)^2.  Returns the
 * loss, the parameter gradient (host, num_params, may be NULL) and y (host, N, may be NULL).
 * Inputs are rounded to BF16 as the network stores them. */
dft_status_t dft_pnet_loss_grad(dft_context* ctx, dft_pnet* net, int nx, int ny, int nz, const float* x,
                                const float* t, double* loss, float* grad, float* y);

typedef struct {
    long coarse_cycles;   /* multigrid cycles spent on the coarse levels */
    int multigrid_cycles; /* V-cycles run */
    double residual;      /* size of the next Jacobi update after them */
    double scale;         /* max |first coarse level's potential|: the network's input/output scale */
} dft_poisson_start_info;

/* Start values for the Jacobi solve of density rho (device): the nested coarse-grid solution
 * (full multigrid over grids of about half the points per axis each) interpolated to g, plus the network's correction when net is not NULL, then up to
 * multigrid_cycles V(2,2) cycles (stopping once the next Jacobi update would be below
 * 0.5e-8).  vstart: device, N doubles, faces zero (grids whose last nodes land on the bounds).
 * info may be NULL. */
dft_status_t dft_poisson_start_dev(dft_context* ctx, const dft_grid* g, dft_pnet* net, const double* rho,
                                   double* vstart, int multigrid_cycles, dft_poisson_start_info* info);

/* calculateHartreePotential from a given start: the interior of vh (device, in/out) is the
 * first iterate, the faces get the reference's boundary values; same stop rule and cap. */
dft_status_t dft_hartree_from_guess_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh,
                                        double tol, long max_sweeps, long* sweeps_out, double* last_diff_out);

/* Seeded synthetic density: kmin..kmax Gaussians with centres uniform in the box, widths
 * uniform in [wmin, wmax] bohr, positive random weights, normalised so sum rho dV is an
 * electron count drawn from ne_min..ne_max (returned in ne_out, may be NULL). */
dft_status_t dft_synthetic_density_dev(dft_context* ctx, const dft_grid* g, unsigned long long seed, int kmin,
                                       int kmax, double wmin, double wmax, int ne_min, int ne_max, double* rho,
                                       int* ne_out);

typedef struct {
    int samples;             /* synthetic densities, each solved to target_tol */
    int validation;          /* of which the last ones are held out */
    int epochs;
    int batch;               /* samples per optimiser step */
    double lr, lr_min;       /* Adam step size, cosine-decayed from lr to lr_min */
    unsigned long long seed;
    double target_tol;       /* Jacobi stop tolerance of the targets (reached via multigrid cycles) */
    long target_max_sweeps;
    int ngrids;              /* 1..4 grids, used in turn */
    dft_grid grids[4];
    int kmin, kmax;          /* Gaussians per density */
    double wmin, wmax;       /* widths (bohr) */
    int ne_min, ne_max;      /* electrons per density */
    int smooth_sweeps;       /* k: the loss adds mean((J^k e)^2), J a Jacobi sweep on the error e */
    double mse_weight;       /* weight of the plain mean(e^2) term */
    int verbose;
} dft_pnet_train_opts;

typedef struct {
    int steps;
    double seconds_data, seconds_train, ms_per_step;
    double mean_target_sweeps;  /* Jacobi sweeps that finished each target after the cycles */
    double train_loss_first_epoch, train_loss_last_epoch;
    double val_loss;         /* network */
    double val_loss_coarse;  /* zero correction: the coarse start alone */
    double* epoch_loss;      /* optional host array, epoch_loss_capacity entries */
    int epoch_loss_capacity;
} dft_pnet_train_report;

/* Trains the network on the device with its own forward, backward and Adam kernels. */
dft_status_t dft_pnet_train_poisson(dft_context* ctx, dft_pnet* net, const dft_pnet_train_opts* opts,
                                    dft_pnet_train_report* report);

/* Learned Davidson preconditioner (replaces the diagonal correction of davidsonCorrection,
 * reference EigenvalueSolverMolecule.cpp:521-555, as dft_eig_opts.preconditioner = -3).  The
 * correction equation (T + sigma) t = r (T = -1/2 lap_h, sigma = max(-theta, 1 Ha)) gets one
 * multigrid cycle, t0, and the network (the same 3-level BF16 U-Net, inputs 2 h^2 r / s and
 * t0 / s with s = max |t0|) adds the remaining correction toward the equation's solution on the
 * interior.  Training pairs come from the plain solver: the residual bands of a block
 * eigensolve (nocc occupied of nbands) in the device potential V on grid g, their targets from
 * opts->target_max_sweeps refined multigrid cycles; opts->samples residual bands are taken
 * (the first opts->validation of them are held out).  report->val_loss is the network's
 * error, report->val_loss_coarse that of the single cycle. */
dft_status_t dft_pnet_train_preconditioner(dft_context* ctx, dft_pnet* net, const dft_grid* g, const double* V,
                                           int nocc, int nbands, const dft_pnet_train_opts* opts,
                                           dft_pnet_train_report* report);

#ifdef __cplusplus
}
#endif
#endif /* DFT_B200_H */
