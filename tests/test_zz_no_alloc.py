"""GPU: the allocation-free Hartree entry point (dft_hartree_noalloc_dev).

It exists for callers that cannot let the library allocate device memory (an application
whose pooled allocator owns the device memory, or a plugin inside its compute step).
Called through the C ABI, it must reproduce dft_hartree_dev exactly (values and sweep
count — the bar the Jacobi solver is held to everywhere) on calls in a row, each on a
different grid so the shared scratch array starts with the previous call's leftovers: one
grid with faces off the bounds (non-zero boundary values), one stopped on an odd sweep
count (the result is then copied back from the array), and one at the 128^3 limit, where
the iterate fills the array up to the control words.  It must reject grids above that
limit with a clear error, and it must allocate nothing: the device's free memory is the
same before and after its calls, in this process and as the first call of a fresh process.

The file is collected last (its name sorts last), so a run that stops at the first failure
has run every other test before this one.
"""
import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import dft_b200
from conftest import gaussian_density

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (grid points, bounds, seed, sweep cap)
CASES = [
    ((24, 22, 20), (-6.0, 6.0, -5.5, 5.5, -5.0, 5.0), 5, 10000),
    ((5, 6, 4), (-2.0, 2.2, -1.0, 1.5, -1.7, 1.3), 6, 10000),  # faces off the bound
    ((40, 36, 32), (-6.0, 6.0, -5.0, 5.0, -4.0, 4.0), 7, 333),  # stops at the odd cap
    ((128, 128, 128), (-12.7, 12.7) * 3, 8, 1001),  # the size limit, odd cap
]


def _solve(lib, ctx, fn, grid, rho_ptr, vh_ptr, max_sweeps):
    sw, last = C.c_long(), C.c_double()
    rc = getattr(lib, fn)(ctx, C.byref(grid), rho_ptr, vh_ptr, 1e-8, max_sweeps, C.byref(sw), C.byref(last))
    assert rc == 0, lib.dft_last_error_message()
    return sw.value, last.value


def test_noalloc_matches_allocating_entry_point(engine):
    import torch

    lib = dft_b200.load()
    odd = False
    for n, b, seed, cap in CASES:  # calls in a row on one context
        na, nb = gaussian_density(n, b, seed)
        g = dft_b200.CartesianGrid(*n, *b).c()
        rho = engine.upload(na + nb)
        v_ref, v_new = engine.array(na.size), engine.array(na.size)
        engine.synchronize()
        free0 = torch.cuda.mem_get_info(engine.device)[0]
        s_new, d_new = _solve(lib, engine.ctx, "dft_hartree_noalloc_dev", g, rho.ptr, v_new.ptr, cap)
        engine.synchronize()
        assert torch.cuda.mem_get_info(engine.device)[0] == free0, "the allocation-free call allocated"
        s_ref, d_ref = _solve(lib, engine.ctx, "dft_hartree_dev", g, rho.ptr, v_ref.ptr, cap)
        assert s_new == s_ref and d_new == d_ref
        assert np.array_equal(v_new.to_host(), v_ref.to_host())
        odd = odd or (s_new % 2 == 1)
    assert odd, "no case ended on an odd sweep count"


FRESH = textwrap.dedent("""
    import ctypes as C, sys
    import numpy as np
    sys.path.insert(0, {root!r})
    sys.path.insert(0, {tests!r})
    import torch
    import dft_b200
    from conftest import gaussian_density
    lib = dft_b200.load()
    eng = dft_b200.Engine(0)
    n, b = (48, 40, 36), (-6.0, 6.0, -5.0, 5.0, -4.5, 4.5)
    na, nb = gaussian_density(n, b, 11)
    g = dft_b200.CartesianGrid(*n, *b).c()
    rho = eng.upload(na + nb)
    v_new, v_ref = eng.array(na.size), eng.array(na.size)
    eng.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    out = []
    for fn, v in (("dft_hartree_noalloc_dev", v_new), ("dft_hartree_noalloc_dev", v_new),
                  ("dft_hartree_dev", v_ref)):
        sw, last = C.c_long(), C.c_double()
        rc = getattr(lib, fn)(eng.ctx, C.byref(g), rho.ptr, v.ptr, 1e-8, 777, C.byref(sw), C.byref(last))
        assert rc == 0, lib.dft_last_error_message()
        eng.synchronize()
        if fn == "dft_hartree_noalloc_dev":
            assert torch.cuda.mem_get_info(0)[0] == free0, "allocated"
        out.append((sw.value, last.value))
    assert out[0] == out[1] == out[2], out
    assert np.array_equal(v_new.to_host(), v_ref.to_host())
    print("fresh-process ok", out[0])
""")


def test_noalloc_first_call_in_fresh_process():
    """The first call of a new process (nothing else has run on the device) allocates
    nothing and matches dft_hartree_dev."""
    code = FRESH.format(root=ROOT, tests=os.path.join(ROOT, "tests"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process ok" in r.stdout


def test_noalloc_rejects_grids_above_limit(engine):
    lib = dft_b200.load()
    g = dft_b200.CartesianGrid(129, 128, 128, -1, 1, -1, 1, -1, 1).c()
    buf = engine.array(16)
    rc = lib.dft_hartree_noalloc_dev(engine.ctx, C.byref(g), buf.ptr, engine.array(16).ptr, 1e-8, 10000, None, None)
    assert rc == dft_b200.DFT_INVALID_ARGUMENT
    assert b"allocation-free" in lib.dft_last_error_message()
