"""CPU: the host eigensolvers of the block Davidson's projected problems (csrc/eigh.cpp).

eigh_lowest computes the lowest m eigenpairs (tridiagonalisation, QL eigenvalues, inverse
iteration with cluster reorthogonalisation, back-transformation).  Checked against numpy on
random, degenerate, tightly clustered, block-split and diagonal matrices: eigenvalues to
1e-12 relative, residuals |A z - w z| and the orthonormality of Z to 1e-10 (eigenvectors of a
degenerate eigenvalue are compared as a subspace, not one by one).
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dft_b200", "csrc")

SHIM = r"""
#include <vector>
#include "eigh.h"
extern "C" int shim_eigh_lowest(int n, const double* a, int m, double* w, double* z) {
    std::vector<double> A(a, a + (size_t)n * n), W, Z;
    if (!dftb::eigh_lowest(n, A, m, W, Z)) return 1;
    for (int j = 0; j < m; ++j) w[j] = W[j];
    for (size_t i = 0; i < (size_t)n * m; ++i) z[i] = Z[i];
    return 0;
}
"""


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("eigh")
    src = d / "shim.cpp"
    src.write_text(SHIM)
    so = d / "libshim.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC, str(src),
                    os.path.join(CSRC, "eigh.cpp"), "-o", str(so)], check=True)
    return C.CDLL(str(so))


def _solve(lib, A, m):
    n = A.shape[0]
    A = np.ascontiguousarray(A, dtype=np.float64)
    w, z = np.zeros(m), np.zeros((n, m))
    dp = C.POINTER(C.c_double)
    rc = lib.shim_eigh_lowest(n, A.ctypes.data_as(dp), m, w.ctypes.data_as(dp), z.ctypes.data_as(dp))
    assert rc == 0
    return w, z


def _check(A, w, z):
    ref = np.linalg.eigvalsh(A)[: len(w)]
    scale = max(np.max(np.abs(ref)), 1.0)
    assert np.max(np.abs(w - ref)) <= 1e-12 * scale * A.shape[0] ** 0.5
    assert np.max(np.abs(A @ z - z * w)) <= 1e-10 * scale
    assert np.max(np.abs(z.T @ z - np.eye(len(w)))) <= 1e-10


def _with_spectrum(lam, seed):
    n = len(lam)
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, n)))
    return (q * lam) @ q.T


@pytest.mark.parametrize("n,m", [(207, 69), (138, 69), (100, 40), (60, 20), (30, 10), (207, 103)])
def test_random(lib, n, m):
    rng = np.random.default_rng(n + m)
    B = rng.standard_normal((n, n))
    A = 0.5 * (B + B.T)
    w, z = _solve(lib, A, m)
    _check(A, w, z)


def test_degenerate_and_clustered(lib):
    n = 150
    lam = np.sort(np.concatenate([
        [-20.0] * 3,                          # exactly triple
        [-5.0, -5.0 + 1e-11, -5.0 + 2e-11],   # cluster far below 1e-3 |A|
        -1.0 + 1e-4 * np.arange(10),          # close but resolvable
        np.linspace(0.0, 50.0, n - 16),
    ]))
    A = _with_spectrum(lam, 3)
    A = 0.5 * (A + A.T)
    w, z = _solve(lib, A, 60)
    _check(A, w, z)


def test_block_split_and_diagonal(lib):
    n = 120
    rng = np.random.default_rng(9)
    A = np.zeros((n, n))
    for s, e in ((0, 40), (40, 41), (41, 90), (90, 120)):  # independent blocks: the tridiagonal splits
        B = rng.standard_normal((e - s, e - s))
        A[s:e, s:e] = 0.5 * (B + B.T)
    A[40, 40] = A[3, 3]
    w, z = _solve(lib, A, 50)
    _check(A, w, z)
    D = np.diag(np.linspace(3.0, -3.0, 80))
    w, z = _solve(lib, D, 30)
    _check(D, w, z)


def test_thick_restart_like_matrix(lib):
    """The Davidson's matrix after a restart: diagonal Ritz block bordered by new rows."""
    k0, k1 = 103, 69
    rng = np.random.default_rng(4)
    n = k0 + k1
    A = np.zeros((n, n))
    A[:k0, :k0] = np.diag(np.sort(rng.uniform(-30, 5, k0)))
    B = 1e-3 * rng.standard_normal((k0, k1))
    C2 = rng.standard_normal((k1, k1))
    A[:k0, k0:] = B
    A[k0:, :k0] = B.T
    A[k0:, k0:] = 0.5 * (C2 + C2.T) + 10.0 * np.eye(k1)
    w, z = _solve(lib, A, 69)
    _check(A, w, z)
