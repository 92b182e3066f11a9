// Dense symmetric eigensolver for the small projected matrices of the block eigensolver
// (k <= a few hundred), in FP64 on the host: Householder reduction to tridiagonal form
// followed by the implicit-shift QL iteration (the classic EISPACK tred2/tql2 pair,
// restated).  The reference diagonalises its (<= 16 x 16) projected matrix by Jacobi
// rotations (EigenvalueSolverMolecule.cpp:290-449); the block method needs all k pairs of
// matrices up to ~200, for which Householder + QL is the O(k^3) choice.
#pragma once

#include <vector>

namespace dftb {

// a: n x n symmetric, row-major (only needs to be symmetric; it is overwritten).
// On return w holds the eigenvalues in ascending order and z (n x n, row-major) the
// orthonormal eigenvectors as columns: z[i*n + j] is component i of eigenvector j.
// Returns false if the QL iteration failed to converge.
bool eigh(int n, std::vector<double>& a, std::vector<double>& w, std::vector<double>& z);

// The lowest m eigenpairs only (1 <= m <= n): w[0..m) ascending, z (n x m, row-major) with
// z[i*m + j] component i of eigenvector j.  Householder tridiagonalisation (all rows, row-major
// loops the compiler vectorises), all eigenvalues of the tridiagonal by QL without vectors,
// eigenvectors of the m lowest by inverse iteration (vectors of eigenvalues closer than
// 1e-3 ||T|| reorthogonalised against each other, as LAPACK's dstein does), then the
// reflectors applied to those m vectors: about 2n^3 + 2n^2 m flops instead of eigh's ~4n^3
// with all n vectors.  Each pair is checked (residual and orthogonality); if a check fails
// the full eigh above decides.  Returns false only if that fails too.
bool eigh_lowest(int n, std::vector<double>& a, int m, std::vector<double>& w, std::vector<double>& z);

}  // namespace dftb
