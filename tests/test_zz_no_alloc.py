"""GPU: the allocation-free Hartree entry point (dft_hartree_noalloc_dev).

It exists for callers that cannot let the library allocate device memory (an application
whose pooled allocator owns the device memory, or a plugin inside its compute step).
Called through the C ABI, it must reproduce dft_hartree_dev exactly (values and sweep
count — the bar the Jacobi solver is held to everywhere) on two calls in a row, the
second on a different grid so the shared scratch array starts with the first call's
leftovers; and it must reject grids above its 128^3 limit with a clear error.

This file is collected last on purpose and also runs alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import dft_b200
from conftest import gaussian_density

pytestmark = pytest.mark.gpu

CASES = [
    ((24, 22, 20), (-6.0, 6.0, -5.5, 5.5, -5.0, 5.0), 5),
    ((5, 6, 4), (-2.0, 2.2, -1.0, 1.5, -1.7, 1.3), 6),  # faces off the bound: non-zero boundary values
]


def _solve(lib, ctx, fn, grid, rho_ptr, vh_ptr):
    sw, last = C.c_long(), C.c_double()
    rc = getattr(lib, fn)(ctx, C.byref(grid), rho_ptr, vh_ptr, 1e-8, 10000, C.byref(sw), C.byref(last))
    assert rc == 0, lib.dft_last_error_message()
    return sw.value, last.value


def test_noalloc_matches_allocating_entry_point(engine):
    lib = dft_b200.load()
    for n, b, seed in CASES:  # two calls in a row
        na, nb = gaussian_density(n, b, seed)
        g = dft_b200.CartesianGrid(*n, *b).c()
        rho = engine.upload(na + nb)
        v_ref, v_new = engine.array(na.size), engine.array(na.size)
        s_ref, d_ref = _solve(lib, engine.ctx, "dft_hartree_dev", g, rho.ptr, v_ref.ptr)
        s_new, d_new = _solve(lib, engine.ctx, "dft_hartree_noalloc_dev", g, rho.ptr, v_new.ptr)
        assert s_new == s_ref and d_new == d_ref
        assert np.array_equal(v_new.to_host(), v_ref.to_host())


def test_noalloc_rejects_grids_above_limit(engine):
    lib = dft_b200.load()
    g = dft_b200.CartesianGrid(129, 128, 128, -1, 1, -1, 1, -1, 1).c()
    buf = engine.array(16)
    rc = lib.dft_hartree_noalloc_dev(engine.ctx, C.byref(g), buf.ptr, engine.array(16).ptr, 1e-8, 10000, None, None)
    assert rc == dft_b200.DFT_INVALID_ARGUMENT
    assert b"allocation-free" in lib.dft_last_error_message()
