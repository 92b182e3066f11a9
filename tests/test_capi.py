"""CPU: the C-ABI library loads and exports every symbol include/dft_b200.h declares;
host-side logic that needs no GPU (option defaults, argument checks before any launch)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dft_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(dft_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("dft_apply_hamiltonian_dev", "dft_hartree_dev", "dft_xc_dev", "dft_solve_orbitals_dev",
                 "dft_scf_molecule", "dft_solve_atoms"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import dft_b200
    lib = dft_b200.load()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding table covers the header
    assert set(declared_symbols()) <= set(dft_b200._SIGS)


def test_defaults_match_reference_constants():
    import dft_b200
    o = dft_b200.default_scf_options()
    assert o.max_iterations == 250 and o.energy_tol == 1e-11 and o.density_tol == 1e-9 and o.ks_tol == 1e-7
    assert o.poisson_tol == 1e-8 and o.poisson_max_sweeps == 10000 and o.eig.tol == 1e-7


def test_errors_without_gpu_are_status_codes():
    """With no usable device the context call fails with a status, not a crash."""
    import dft_b200
    lib = dft_b200.load()
    p = ctypes.c_void_p()
    rc = lib.dft_context_create(9999, ctypes.byref(p))
    assert rc != 0
    assert lib.dft_last_error_message()


def test_grid_validation_mirrors_reference():
    import dft_b200
    with pytest.raises(ValueError, match="two points"):
        dft_b200.CartesianGrid(1, 4, 4, 0, 1, 0, 1, 0, 1)
    with pytest.raises(ValueError, match="bounds"):
        dft_b200.CartesianGrid(4, 4, 4, 1, 0, 0, 1, 0, 1)
    with pytest.raises(ValueError):
        dft_b200.Molecule().addNucleus(0, 0, 0, 0)
