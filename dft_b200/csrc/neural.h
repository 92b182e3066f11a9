// Learned start for the Jacobi Poisson solve (no counterpart in the reference, whose solve
// always starts from zero, HartreePotentialMolecule.cpp:152-155).
//
// The start is built in two parts.  A coarse grid with the same bounds and about a quarter
// of the points per axis carries the long-range part: the density is restricted to it with
// the transposed trilinear weights (charge-conserving), solved there with the same Jacobi
// kernels, and interpolated back trilinearly.  A small 3D convolutional network (a 3-level
// U-Net, BF16 activations, FP32 accumulation) then predicts the short-range correction from
// the density and the interpolated coarse potential.  The fine Jacobi solve starts from the
// sum and runs with the unchanged stop rule, so the answer is the Jacobi answer; only the
// number of sweeps (or, at the sweep cap, the remaining error) changes.
#pragma once

#include "common.cuh"

struct dft_pnet;

namespace dftb {

struct PoissonGuessInfo {
    long coarse_cycles = 0;  // multigrid cycles spent on the coarse levels
    int coarse_n[3] = {0, 0, 0};
    double scale = 0.0;  // max |coarse potential|, the network's input/output scale
    int cycles = 0;      // multigrid V-cycles run
    double residual = 0.0;  // size of the next Jacobi update after them
};

// Coarse points per axis for a fine axis of n points (about half).
int coarse_points(int n);

// Nested coarse-grid start (poisson_start.cu): vup = the interpolated solution of the coarse
// levels; *scale_dev = max |first coarse level's solution| on the device.  slab holds
// coarse_slab_doubles(g) doubles.  Returns the multigrid cycles spent on the coarse levels.
size_t coarse_slab_doubles(const Grid& g);
long coarse_start(dft_context* ctx, double* slab, const Grid& g, const double* rho, double* vup, double** scale_dev);

// Multigrid V(2,2) cycles on v in place (faces held at their values, coarse corrections zero
// on faces) until the next Jacobi update would be below tol or max_cycles ran.  Returns the
// cycles run.
int multigrid(dft_context* ctx, const Grid& g, const double* rho, double* v, double tol, int max_cycles,
              double* resid_out);

// Start values for the Jacobi solve: nested coarse start, plus the network's correction when
// net is not null, then up to `cycles` multigrid cycles.  out: N doubles (faces zero).
void poisson_start(dft_context* ctx, dft_pnet* net, const Grid& g, const double* rho, double* out, int cycles,
                   PoissonGuessInfo* info);

// Adds the network's correction to the coarse start v (neural.cu).
void pnet_correct(dft_context* ctx, dft_pnet* net, const Grid& g, const double* rho, double* v,
                  const double* scale_dev);

dft_pnet* pnet_create(dft_context* ctx, int in_channels, unsigned long long seed);
void pnet_destroy(dft_pnet* net);
size_t pnet_num_params(const dft_pnet* net);
void pnet_get_params(dft_context* ctx, dft_pnet* net, float* host);
void pnet_set_params(dft_context* ctx, dft_pnet* net, const float* host);

// One forward + backward pass on a volume (nx, ny, nz) with host input x[N][in_channels]
// and target t[N] (loss = mean over interior points of (y - t)^2).  Outputs the loss,
// the gradient with respect to every parameter (host, nparams) and the prediction y (host, N).
void pnet_loss_grad(dft_context* ctx, dft_pnet* net, int nx, int ny, int nz, const float* x_host,
                    const float* t_host, double* loss, float* grad_host, float* y_host);

// Seeded synthetic density: 1-8 Gaussians, centres uniform in the box, widths uniform in
// [wmin, wmax], positive amplitudes, normalised to an integer electron count in [ne_min, ne_max].
// Returns the electron count.
int synthetic_density(dft_context* ctx, const Grid& g, unsigned long long seed, int kmin, int kmax, double wmin,
                      double wmax, int ne_min, int ne_max, double* rho);

void pnet_train_poisson(dft_context* ctx, dft_pnet* net, const dft_pnet_train_opts* opts,
                        dft_pnet_train_report* report);

// Learned Davidson preconditioner: T_a (the multigrid cycle's t0 for band active[a] of R) gets
// the network's correction toward the solution of (T + sigma) t = r on the interior.
void pnet_precondition(dft_context* ctx, dft_pnet* net, const Grid& g, const double* R, long long ld,
                       const int* active, int na, double* T);
// Trains it on residual bands that the plain eigensolver (multigrid preconditioner) produces in
// the potential V (device), targets from opts->target_max_sweeps refined multigrid cycles.
void pnet_train_precond(dft_context* ctx, dft_pnet* net, const Grid& g, const double* V, int nocc, int nbands,
                        const dft_pnet_train_opts* opts, dft_pnet_train_report* report);

}  // namespace dftb
