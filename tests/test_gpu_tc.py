"""GPU: the tensor-core (tcgen05, TF32 hi+lo) Gram product and the mixed-precision eigensolver.

Bars: the TF32 hi+lo Gram matches FP64 to 1e-4 of the largest |entry| (FP32 accumulation in
TMEM over chunks of <= 8192 points: sums of same-sign terms lose ~6.5e-5 of their size at 96^3,
measured, growing with the chunk length, not with N); the mixed-precision eigensolver, which switches to FP64 before its
final iterations, gives the FP64 eigenvalues to 1e-9 Ha.
"""
import numpy as np
import pytest

import dft_b200
from oracle.bindings import PZ81  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[(0, 0), (1, 0), (0, 1)], ids=["regs", "ring", "tma"])
def tc_ring(request, engine):
    """The staging variants of the tensor-core Gram product (register prefetch, cp.async ring,
    TMA ring); shapes a variant does not take (odd leading dimension, > 128 columns for the
    cp.async ring) fall back."""
    engine.set_tuning("tensor_core_ring", request.param[0])
    engine.set_tuning("tensor_core_tma", request.param[1])
    yield request.param
    engine.set_tuning("tensor_core_ring", 0)
    engine.set_tuning("tensor_core_tma", 0)


@pytest.mark.parametrize("ka,kb,n", [(12, 12, (40, 40, 40)), (50, 70, (64, 48, 33)), (130, 300, (32, 32, 40)),
                                     (200, 69, (48, 48, 48)), (1, 3, (5, 7, 9)), (129, 127, (33, 29, 41)),
                                     (207, 69, (96, 96, 96))])
def test_gram_tensor_cores_vs_fp64(engine, ka, kb, n, tc_ring):
    g = dft_b200.CartesianGrid(*n, -3.0, 3.0, -2.0, 2.5, -1.5, 1.7)
    N = g.getSize()
    rng = np.random.default_rng(ka * 1000 + kb)
    A = rng.standard_normal((ka, N))
    B = A[: min(ka, kb)].copy() if kb <= ka else rng.standard_normal((kb, N))
    B = B if B.shape[0] == kb else rng.standard_normal((kb, N))
    dA, dB = engine.upload(A), engine.upload(B)
    c64 = engine.gram(g, dA, N, ka, dB, N, kb, precision=0)
    ctc = engine.gram(g, dA, N, ka, dB, N, kb, precision=1)
    dV = g.getDx() * g.getDy() * g.getDz()
    ref = A @ B.T * dV
    assert np.max(np.abs(c64 - ref)) < 1e-10 * np.max(np.abs(ref))
    assert np.max(np.abs(ctc - c64)) < 1e-4 * np.max(np.abs(c64))


def test_mixed_precision_eigensolver(engine, port, tc_ring):
    n, b = (32, 30, 28), (-5.0, 5.0, -4.6, 4.6, -4.2, 4.2)
    g = dft_b200.CartesianGrid(*n, *b)
    N = g.getSize()
    Z, xyz = [8, 1, 1], np.array([0.05, 0.07, 0.03, 1.43, 0.07, 1.1, -1.43, 0.07, 1.1])
    V = port.nuclear_potential(n, b, Z, xyz)
    res = {}
    for mixed in (0, 1):
        psi = engine.array(8 * N)
        eig, it = engine.solve_orbitals(g, engine.upload(V), 5, 8, psi, N, mixed_precision=mixed)
        res[mixed] = eig
    assert np.max(np.abs(res[1][:5] - res[0][:5])) < 1e-9


@pytest.mark.parametrize("k,m,n", [(40, 12, (40, 40, 40)), (207, 69, (33, 30, 28)), (64, 300, (20, 21, 22)),
                                   (5, 3, (7, 9, 11))])
def test_rotation_tensor_cores_vs_fp64(engine, k, m, n):
    g = dft_b200.CartesianGrid(*n, -3.0, 3.0, -2.0, 2.5, -1.5, 1.7)
    N = g.getSize()
    rng = np.random.default_rng(k * 7 + m)
    V = rng.standard_normal((k, N))
    Y = rng.standard_normal((k, m))
    dV = engine.upload(V)
    X64, Xtc = engine.array(m * N), engine.array(m * N)
    engine.rotate(g, dV, N, k, Y, X64, N, precision=0)
    engine.rotate(g, dV, N, k, Y, Xtc, N, precision=1)
    ref = Y.T @ V
    a, b = X64.to_host((m, N)), Xtc.to_host((m, N))
    assert np.max(np.abs(a - ref)) < 1e-11 * np.max(np.abs(ref))
    assert np.max(np.abs(b - a)) < 2e-6 * np.max(np.abs(a))


def test_gram_ring_padded_rows_odd_points(engine):
    """Odd point count with an even leading dimension: the cp.async ring's last 16-byte chunk
    carries one point and a NaN in the padding, which must not be read; the TMA map ends at the
    last point (the copy zero-fills past it)."""
    n = (33, 29, 41)
    g = dft_b200.CartesianGrid(*n, -3.0, 3.0, -2.0, 2.5, -1.5, 1.7)
    N = g.getSize()
    assert N % 2 == 1
    ld = N + 1
    rng = np.random.default_rng(7)
    A = np.full((20, ld), np.nan)
    B = np.full((24, ld), np.nan)
    A[:, :N] = rng.standard_normal((20, N))
    B[:, :N] = rng.standard_normal((24, N))
    dA, dB = engine.upload(A), engine.upload(B)
    c64 = engine.gram(g, dA, ld, 20, dB, ld, 24, precision=0)
    for key in ("tensor_core_ring", "tensor_core_tma"):
        try:
            engine.set_tuning(key, 1)
            ctc = engine.gram(g, dA, ld, 20, dB, ld, 24, precision=1)
        finally:
            engine.set_tuning(key, 0)
        assert np.all(np.isfinite(ctc)), key
        assert np.max(np.abs(ctc - c64)) < 1e-5 * np.max(np.abs(c64)), key
