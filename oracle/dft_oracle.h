/*
 * TEST INFRASTRUCTURE — the CPU oracle.  A plain-C restatement of the reference
 * (willandru/DFT) algorithms on the GPU hot path, used by tests/, by
 * __graft_entry__.smoke() and by the CPU-baseline legs of bench.py as the checker.
 * The product (dft_b200/) never links, loads or calls it.
 *
 * Parity pin: every entry point below is checked against the reference's own
 * sources compiled into oracle/_ref/libdft_ref.so (tests/test_oracle_pin.py) and
 * against the README golden energies (tests/golden/radial_ref.json).
 *
 * Conventions mirror the reference: grids are n[3] = {nx,ny,nz} and
 * b[6] = {xmin,xmax,ymin,ymax,zmin,zmax} (CartesianGrid.cpp:5-48), point index
 * (k*ny + j)*nx + i, band blocks are band-major (band b at psi + b*N).
 * kind: 0 = PZ81, 1 = PBE96.  Every function returns 0 on success and non-zero
 * with oracle_last_error() set where the reference throws.
 */
#ifndef DFT_ORACLE_H
#define DFT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

const char* oracle_last_error(void);

int oracle_xc_evaluate(int kind, long m, const double* na, const double* nb, const double* ga,
                       const double* gb, double* out5);

int oracle_apply_hamiltonian(const long* n, const double* b, const double* V, const double* psi, double* out);
int oracle_hartree_potential(const long* n, const double* b, const double* rho, double* out);
int oracle_hartree_potential_ex(const long* n, const double* b, const double* rho, double* out, long* sweeps,
                                double* last_diff);
int oracle_hartree_energy(const long* n, const double* b, const double* rho, const double* vh, double* e);
int oracle_xc_potential(int kind, const long* n, const double* b, const double* na, const double* nb, int spin,
                        double* out);
int oracle_xc_energy(int kind, const long* n, const double* b, const double* na, const double* nb, double* e);
int oracle_nuclear_potential(const long* n, const double* b, int nnuc, const int* Z, const double* xyz,
                             double* out);
int oracle_nuclear_repulsion(int nnuc, const int* Z, const double* xyz, double* e);
int oracle_kinetic_energy(const long* n, const double* b, int nbands, const double* psi, const int* electrons,
                          double* e);
int oracle_spin_density(long N, int nbands, const double* psi, const int* electrons, double* out);
int oracle_density_difference(const long* n, const double* b, const double* old_d, const double* new_d,
                              double* out);
int oracle_ks_residual(const long* n, const double* b, const double* V, int nbands, const double* psi,
                       const double* eig, double* out);
int oracle_solve_orbitals(const long* n, const double* b, const double* V, int norb, const double* init,
                          double* psi_out, double* eig_out);
int oracle_scf_molecule(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int charge,
                        int multiplicity, int kind, double* energies6, double* stats4, int n_eig,
                        double* eig_out, double* dens_out);

int oracle_scf_sample(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int multiplicity,
                      int kind, int iterations, double* seconds2);

int oracle_solve_atom(int Z, int kind, long points, double rmax, double* energies5, double* stats4, int n_eig,
                      double* eig_out, int* n_eig_written);
int oracle_radial_hartree(long points, double rmax, const double* rho, double* out);
int oracle_radial_xc_potential(int kind, long points, double rmax, const double* na, const double* nb, int spin,
                               double* out);
int oracle_radial_xc_energy(int kind, long points, double rmax, const double* na, const double* nb, double* e);
int oracle_radial_solve_orbital(long points, double rmax, const double* veff, int l, int index, double* eig,
                                double* u_out);
int oracle_radial_sturm_count(long points, double rmax, const double* veff, int l, double energy, long* count);
int oracle_atomic_configuration(int Z, int cap, int* rows, int* nrows);

#ifdef __cplusplus
}
#endif
#endif
