"""dft_b200 — B200-native real-space Kohn–Sham engine, Python face.

The compute path is libdft_b200.so (CUDA, sm_100a) behind the C ABI in
include/dft_b200.h; this module only marshals arguments through ctypes.  There is no CPU
fallback: importing works anywhere, but every call raises if the library or a GPU is
missing.

Two layers are exported:

* ``Engine`` — thin, device-pointer-level access to each C entry point (tests, benchmarks).
* Reference-named functions mirroring the reference's C++ driver API
  (``solveMolecularSelfConsistentField``, ``solveAtom``, ``applyMolecularKohnShamHamiltonian``,
  ``calculateHartreePotential`` ...), taking and returning host numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdft_b200.so")

# ----------------------------------------------------------------- C types -------------
DFT_OK, DFT_INVALID_ARGUMENT, DFT_NOT_CONVERGED, DFT_CAP_REACHED, DFT_SINGULAR, DFT_CUDA_ERROR, DFT_NUMERICAL = range(7)
PZ81_KIND, PBE96_KIND = 0, 1


class dft_grid(C.Structure):
    _fields_ = [("nx", C.c_long), ("ny", C.c_long), ("nz", C.c_long),
                ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double),
                ("ymax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double)]


class dft_eig_opts(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iterations", C.c_int), ("max_subspace", C.c_int), ("verbose", C.c_int),
                ("preconditioner", C.c_int), ("mixed_precision", C.c_int), ("preconditioner_net", C.c_void_p)]


class dft_scf_opts(C.Structure):
    _fields_ = [("max_iterations", C.c_int), ("energy_tol", C.c_double), ("density_tol", C.c_double),
                ("ks_tol", C.c_double), ("stop_abs_de", C.c_double), ("poisson_tol", C.c_double),
                ("poisson_max_sweeps", C.c_long), ("extra_bands", C.c_int), ("eig", dft_eig_opts),
                ("verbose", C.c_int), ("poisson_start", C.c_int), ("poisson_net", C.c_void_p), ("mixer", C.c_int),
                ("pulay_depth", C.c_int), ("pulay_beta", C.c_double), ("adaptive_eig_tol", C.c_int),
                ("smearing_kt", C.c_double), ("kerker_q0", C.c_double),
                ("stop_abs_deig", C.c_double), ("log_path", C.c_char_p), ("autotune", C.c_int),
                ("initial_density", C.c_int),
                ("hartree_boundary", C.c_int), ("poisson_predict", C.c_int),
                ("poisson_fixed_point", C.c_int), ("stop_abs_drho", C.c_double)]


class dft_autotune_report(C.Structure):
    _fields_ = [("hpsi_bands_per_thread", C.c_int), ("hpsi_ms", C.c_double * 3),
                ("jacobi_sweeps_per_launch", C.c_int), ("jacobi_us_per_sweep", C.c_double * 6),
                ("cached", C.c_int), ("hpsi_variant", C.c_int), ("hpsi_tma_ms", C.c_double * 4),
                ("hpsi_prefetch_ms", C.c_double), ("hpsi_zchunk", C.c_int), ("hpsi_zchunk_ms", C.c_double * 5)]


# dft_poisson_start
POISSON_COLD, POISSON_PREVIOUS, POISSON_NETWORK, POISSON_COARSE, POISSON_HYBRID, POISSON_MULTIGRID = 0, 1, 2, 3, 4, 5


class dft_poisson_start_info(C.Structure):
    _fields_ = [("coarse_cycles", C.c_long), ("multigrid_cycles", C.c_int), ("residual", C.c_double),
                ("scale", C.c_double)]


class dft_pnet_train_opts(C.Structure):
    _fields_ = [("samples", C.c_int), ("validation", C.c_int), ("epochs", C.c_int), ("batch", C.c_int),
                ("lr", C.c_double), ("lr_min", C.c_double), ("seed", C.c_ulonglong), ("target_tol", C.c_double),
                ("target_max_sweeps", C.c_long), ("ngrids", C.c_int), ("grids", dft_grid * 4), ("kmin", C.c_int),
                ("kmax", C.c_int), ("wmin", C.c_double), ("wmax", C.c_double), ("ne_min", C.c_int),
                ("ne_max", C.c_int), ("smooth_sweeps", C.c_int), ("mse_weight", C.c_double), ("verbose", C.c_int)]


class dft_pnet_train_report(C.Structure):
    _fields_ = [("steps", C.c_int), ("seconds_data", C.c_double), ("seconds_train", C.c_double),
                ("ms_per_step", C.c_double), ("mean_target_sweeps", C.c_double),
                ("train_loss_first_epoch", C.c_double), ("train_loss_last_epoch", C.c_double),
                ("val_loss", C.c_double), ("val_loss_coarse", C.c_double), ("epoch_loss", C.POINTER(C.c_double)),
                ("epoch_loss_capacity", C.c_int)]


class dft_scf_iteration(C.Structure):
    _fields_ = [("iteration", C.c_int), ("energy", C.c_double), ("energy_difference", C.c_double),
                ("density_difference", C.c_double), ("ks_residual", C.c_double), ("mixing", C.c_double),
                ("poisson_sweeps_in", C.c_long), ("poisson_sweeps_out", C.c_long),
                ("eig_iterations_alpha", C.c_int), ("eig_iterations_beta", C.c_int),
                ("ms_hartree", C.c_double), ("ms_xc", C.c_double), ("ms_orbitals", C.c_double),
                ("ms_density", C.c_double), ("ms_energy", C.c_double), ("ms_total", C.c_double),
                ("eigenvalue_difference", C.c_double), ("poisson_cycles_in", C.c_int),
                ("poisson_cycles_out", C.c_int)]


class dft_scf_result(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("external", C.c_double), ("hartree", C.c_double),
                ("exchange_correlation", C.c_double), ("nuclear_repulsion", C.c_double), ("total", C.c_double),
                ("iterations", C.c_int), ("converged", C.c_int), ("density_difference", C.c_double),
                ("energy_difference", C.c_double), ("max_ks_residual", C.c_double), ("n_alpha", C.c_int),
                ("n_beta", C.c_int), ("eigenvalues", C.POINTER(C.c_double)),
                ("alpha_density", C.POINTER(C.c_double)), ("beta_density", C.POINTER(C.c_double)),
                ("alpha_potential", C.POINTER(C.c_double)), ("beta_potential", C.POINTER(C.c_double)),
                ("orbitals", C.POINTER(C.c_double)),
                ("history", C.POINTER(dft_scf_iteration)), ("history_capacity", C.c_int),
                ("history_len", C.c_int), ("seconds", C.c_double),
                ("last_energy_criterion_iteration", C.c_int), ("last_density_criterion_iteration", C.c_int),
                ("last_ks_criterion_iteration", C.c_int), ("min_energy_difference", C.c_double),
                ("min_density_difference", C.c_double), ("min_ks_residual", C.c_double),
                ("final_mixing", C.c_double)]


class dft_atom_result(C.Structure):
    _fields_ = [("Z", C.c_int), ("kind", C.c_int), ("kinetic", C.c_double), ("external", C.c_double),
                ("hartree", C.c_double), ("exchange_correlation", C.c_double), ("total", C.c_double),
                ("iterations", C.c_int), ("converged", C.c_int), ("density_difference", C.c_double),
                ("max_ks_residual", C.c_double), ("n_orbitals", C.c_int), ("eigenvalues", C.c_double * 16),
                ("status", C.c_int)]


# exported symbols and their argument types (checked by the CPU symbol test)
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_SIGS = {
    "dft_last_error_message": ([], C.c_char_p),
    "dft_version": ([], C.c_char_p),
    "dft_context_create": ([C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "dft_context_destroy": ([_P], C.c_int),
    "dft_context_synchronize": ([_P], C.c_int),
    "dft_context_set_tuning": ([_P, C.c_char_p, C.c_long], C.c_int),
    "dft_context_stream": ([_P], C.c_void_p),
    "dft_autotune": ([_P, C.POINTER(dft_grid), C.c_int, C.POINTER(dft_autotune_report)], C.c_int),
    "dft_context_launch_count": ([_P], C.c_longlong),
    "dft_context_counter": ([_P, C.c_char_p], C.c_longlong),
    "dft_device_alloc": ([_P, C.c_size_t, C.POINTER(C.c_void_p)], C.c_int),
    "dft_device_free": ([_P, _P], C.c_int),
    "dft_copy_h2d": ([_P, _P, _P, C.c_size_t], C.c_int),
    "dft_copy_d2h": ([_P, _P, _P, C.c_size_t], C.c_int),
    "dft_apply_hamiltonian_dev": ([_P, C.POINTER(dft_grid), _P, _P, _P, C.c_int, C.c_long], C.c_int),
    "dft_hartree_dev": ([_P, C.POINTER(dft_grid), _P, _P, C.c_double, C.c_long, C.POINTER(C.c_long), _D], C.c_int),
    "dft_hartree_noalloc_dev": ([_P, C.POINTER(dft_grid), _P, _P, C.c_double, C.c_long, C.POINTER(C.c_long), _D],
                                C.c_int),
    "dft_hartree_monopole_dev": ([_P, C.POINTER(dft_grid), _P, _P, C.c_double, C.c_long, C.POINTER(C.c_long), _D],
                                 C.c_int),
    "dft_hartree_energy_dev": ([_P, C.POINTER(dft_grid), _P, _P, _D], C.c_int),
    "dft_zslab_jacobi_init_dev": ([_P, C.POINTER(dft_grid), C.c_int, C.c_int, C.c_double, _P, _P], C.c_int),
    "dft_zslab_jacobi_sweeps_dev": ([_P, C.POINTER(dft_grid), C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P,
                                     C.c_int, _P], C.c_int),
    "dft_zslab_hamiltonian_dev": ([_P, C.POINTER(dft_grid), C.c_int, C.c_int, _P, _P, _P, C.c_int, C.c_long],
                                  C.c_int),
    "dft_zslab_xc_dev": ([_P, C.POINTER(dft_grid), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _D],
                         C.c_int),
    "dft_zslab_gram_dev": ([_P, C.POINTER(dft_grid), C.c_int, C.c_int, C.c_int, C.c_int, _P, C.c_long, C.c_int, _P,
                           C.c_long, C.c_int, C.c_int, _D], C.c_int),
    "dft_xc_dev": ([_P, C.POINTER(dft_grid), C.c_int, _P, _P, _P, _P, _D], C.c_int),
    "dft_xc_evaluate_dev": ([_P, C.c_int, C.c_long, _P, _P, _P, _P, _P], C.c_int),
    "dft_spin_density_dev": ([_P, C.c_long, _P, C.c_int, C.c_long, _D, _P], C.c_int),
    "dft_kinetic_energy_dev": ([_P, C.POINTER(dft_grid), _P, C.c_int, C.c_long, _D, _D], C.c_int),
    "dft_nuclear_potential_dev": ([_P, C.POINTER(dft_grid), C.c_int, C.POINTER(C.c_int), _D, _P], C.c_int),
    "dft_solve_orbitals_dev": ([_P, C.POINTER(dft_grid), _P, C.c_int, C.c_int, _P, C.c_long, C.c_int, _D,
                                C.POINTER(dft_eig_opts), C.POINTER(C.c_int)], C.c_int),
    "dft_rotate_dev": ([_P, C.POINTER(dft_grid), _P, C.c_long, C.c_int, _D, C.c_int, _P, C.c_long, C.c_int],
                       C.c_int),
    "dft_screened_poisson_dev": ([_P, C.POINTER(dft_grid), _P, _P, C.c_double, C.c_int], C.c_int),
    "dft_gram_dev": ([_P, C.POINTER(dft_grid), _P, C.c_long, C.c_int, _P, C.c_long, C.c_int, C.c_int, _D], C.c_int),
    "dft_scf_default_options": ([C.POINTER(dft_scf_opts)], None),
    "dft_scf_molecule": ([_P, C.POINTER(dft_grid), C.c_int, C.POINTER(C.c_int), _D, C.c_int, C.c_int, C.c_int,
                          C.POINTER(dft_scf_opts), C.POINTER(dft_scf_result)], C.c_int),
    "dft_solve_atoms": ([_P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_long, C.c_double,
                         C.POINTER(dft_atom_result)], C.c_int),
    "dft_hartree_from_guess_dev": ([_P, C.POINTER(dft_grid), _P, _P, C.c_double, C.c_long, C.POINTER(C.c_long),
                                    _D], C.c_int),
    "dft_pnet_create": ([_P, C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p)], C.c_int),
    "dft_pnet_destroy": ([_P], C.c_int),
    "dft_pnet_num_params": ([_P, C.POINTER(C.c_size_t)], C.c_int),
    "dft_pnet_get_params": ([_P, _P, C.POINTER(C.c_float), C.c_size_t], C.c_int),
    "dft_pnet_set_params": ([_P, _P, C.POINTER(C.c_float), C.c_size_t], C.c_int),
    "dft_pnet_loss_grad": ([_P, _P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), _D,
                            C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
    "dft_poisson_start_dev": ([_P, C.POINTER(dft_grid), _P, _P, _P, C.c_int, C.POINTER(dft_poisson_start_info)],
                              C.c_int),
    "dft_synthetic_density_dev": ([_P, C.POINTER(dft_grid), C.c_ulonglong, C.c_int, C.c_int, C.c_double,
                                   C.c_double, C.c_int, C.c_int, _P, C.POINTER(C.c_int)], C.c_int),
    "dft_pnet_train_poisson": ([_P, _P, C.POINTER(dft_pnet_train_opts), C.POINTER(dft_pnet_train_report)],
                               C.c_int),
    "dft_pnet_train_preconditioner": ([_P, _P, C.POINTER(dft_grid), _P, C.c_int, C.c_int,
                                       C.POINTER(dft_pnet_train_opts), C.POINTER(dft_pnet_train_report)], C.c_int),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libdft_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m dft_b200.build`")
    lib = C.CDLL(path)
    for name, (args, res) in _SIGS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


class DFTError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


def _check(rc: int) -> None:
    if rc != DFT_OK:
        raise DFTError(rc, load().dft_last_error_message().decode(errors="replace"))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ----------------------------------------------------------------- grids & inputs -------
class CartesianGrid:
    """reference CartesianGrid (CartesianGrid.h:5-60): node-centred, spacing (max-min)/(n-1)."""

    def __init__(self, nx, ny, nz, xmin, xmax, ymin, ymax, zmin, zmax):
        if nx < 2 or ny < 2 or nz < 2:
            raise ValueError("CartesianGrid requires at least two points per dimension.")
        if xmax <= xmin or ymax <= ymin or zmax <= zmin:
            raise ValueError("CartesianGrid requires valid spatial bounds.")
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.bounds = (float(xmin), float(xmax), float(ymin), float(ymax), float(zmin), float(zmax))

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    def getSize(self) -> int:
        return self.nx * self.ny * self.nz

    def getDx(self):
        return (self.bounds[1] - self.bounds[0]) / (self.nx - 1)

    def getDy(self):
        return (self.bounds[3] - self.bounds[2]) / (self.ny - 1)

    def getDz(self):
        return (self.bounds[5] - self.bounds[4]) / (self.nz - 1)

    def c(self) -> dft_grid:
        return dft_grid(self.nx, self.ny, self.nz, *self.bounds)


class RadialGrid:
    """reference RadialGrid (RadialGrid.h:6-18): r_i = (i+1) rMax/(points+1)."""

    def __init__(self, points: int = 2000, rmax: float = 30.0):
        if points <= 0:
            raise ValueError("El numero de puntos debe ser mayor que cero.")
        if rmax <= 0:
            raise ValueError("RMAX debe ser mayor que cero.")
        self.points, self.rmax = int(points), float(rmax)

    def coordinates(self) -> np.ndarray:
        return (np.arange(self.points) + 1.0) * (self.rmax / (self.points + 1))


class Molecule:
    """reference Molecule (Molecule.h:6-35)."""

    def __init__(self, charge: int = 0):
        self.charge = int(charge)
        self.nuclei: List[tuple] = []

    def addNucleus(self, atomicNumber: int, x: float, y: float, z: float) -> None:
        if atomicNumber <= 0:
            raise ValueError("Atomic number must be greater than zero.")
        self.nuclei.append((int(atomicNumber), float(x), float(y), float(z)))

    def getCharge(self) -> int:
        return self.charge

    def getElectronCount(self) -> int:
        return sum(n[0] for n in self.nuclei) - self.charge

    def arrays(self):
        Z = np.array([n[0] for n in self.nuclei], dtype=np.int32)
        xyz = np.array([n[1:] for n in self.nuclei], dtype=np.float64).reshape(-1)
        return Z, xyz


class XCFunctional:
    kind: int = -1


class PZ81(XCFunctional):
    kind = PZ81_KIND


class PBE96(XCFunctional):
    kind = PBE96_KIND


def _kind(f) -> int:
    if isinstance(f, XCFunctional):
        return f.kind
    if isinstance(f, str):
        return {"PZ81": PZ81_KIND, "PBE96": PBE96_KIND}[f.upper()]
    return int(f)


# ----------------------------------------------------------------- engine ---------------
class DeviceArray:
    """A float64 device buffer owned by an Engine (no torch dependency)."""

    def __init__(self, eng: "Engine", n: int):
        self.eng, self.n = eng, int(n)
        p = C.c_void_p()
        _check(load().dft_device_alloc(eng.ctx, max(self.n, 1) * 8, C.byref(p)))
        self.ptr = p.value

    @classmethod
    def from_host(cls, eng, a) -> "DeviceArray":
        a = np.ascontiguousarray(a, dtype=np.float64)
        d = cls(eng, a.size)
        _check(load().dft_copy_h2d(eng.ctx, d.ptr, a.ctypes.data, a.size * 8))
        return d

    def to_host(self, shape=None) -> np.ndarray:
        out = np.empty(self.n)
        _check(load().dft_copy_d2h(self.eng.ctx, out.ctypes.data, self.ptr, self.n * 8))
        return out.reshape(shape) if shape is not None else out

    def free(self):
        if self.ptr:
            _check(load().dft_device_free(self.eng.ctx, self.ptr))
            self.ptr = None

    def __del__(self):
        try:
            if self.ptr and self.eng.ctx:
                load().dft_device_free(self.eng.ctx, self.ptr)
        except Exception:
            pass


class Engine:
    """One dft_context on one GPU."""

    def __init__(self, device: int = 0):
        lib = load()
        p = C.c_void_p()
        _check(lib.dft_context_create(device, C.byref(p)))
        self.ctx = p.value
        self.device = device

    def close(self):
        if self.ctx:
            load().dft_context_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def synchronize(self):
        _check(load().dft_context_synchronize(self.ctx))

    def set_tuning(self, key: str, value: int):
        _check(load().dft_context_set_tuning(self.ctx, key.encode(), int(value)))

    @property
    def stream(self) -> int:
        return load().dft_context_stream(self.ctx)

    @property
    def launches(self) -> int:
        return load().dft_context_launch_count(self.ctx)

    def autotune(self, grid, nbands: int) -> dict:
        """Times the bit-identical launch variants on this grid and keeps the fastest."""
        g = grid.c()
        r = dft_autotune_report()
        _check(load().dft_autotune(self.ctx, C.byref(g), int(nbands), C.byref(r)))
        return {"hpsi_bands_per_thread": r.hpsi_bands_per_thread, "hpsi_ms": list(r.hpsi_ms),
                "jacobi_sweeps_per_launch": r.jacobi_sweeps_per_launch,
                "jacobi_us_per_sweep": list(r.jacobi_us_per_sweep), "cached": bool(r.cached),
                "hpsi_variant": r.hpsi_variant, "hpsi_tma_ms": list(r.hpsi_tma_ms),
                "hpsi_prefetch_ms": r.hpsi_prefetch_ms, "hpsi_zchunk": r.hpsi_zchunk,
                "hpsi_zchunk_ms": list(r.hpsi_zchunk_ms)}

    def counter(self, name: str) -> int:
        return load().dft_context_counter(self.ctx, name.encode())

    def array(self, n) -> DeviceArray:
        return DeviceArray(self, n)

    def upload(self, a) -> DeviceArray:
        return DeviceArray.from_host(self, a)

    # --- device-pointer entry points ------------------------------------------------
    def apply_hamiltonian(self, grid: CartesianGrid, V, psi, hpsi, nbands: int, ld: int):
        g = grid.c()
        _check(load().dft_apply_hamiltonian_dev(self.ctx, C.byref(g), _ptr(V), _ptr(psi), _ptr(hpsi), nbands, ld))

    def hartree(self, grid, rho, vh, tol=1e-8, max_sweeps=10000):
        g = grid.c()
        sw = C.c_long()
        ld = C.c_double()
        _check(load().dft_hartree_dev(self.ctx, C.byref(g), _ptr(rho), _ptr(vh), tol, max_sweeps, C.byref(sw),
                                      C.byref(ld)))
        return sw.value, ld.value

    def hartree_monopole(self, grid, rho, vh, tol=1e-8, max_sweeps=10000):
        """Hartree potential with Q/|r| on every face (dft_scf_opts.hartree_boundary = 1)."""
        g = grid.c()
        sw = C.c_long()
        ld = C.c_double()
        _check(load().dft_hartree_monopole_dev(self.ctx, C.byref(g), _ptr(rho), _ptr(vh), tol, max_sweeps,
                                               C.byref(sw), C.byref(ld)))
        return sw.value, ld.value

    def hartree_from_guess(self, grid, rho, vh, tol=1e-8, max_sweeps=10000):
        """Jacobi from the interior of vh (in/out) with the reference's stop rule."""
        g = grid.c()
        sw = C.c_long()
        ld = C.c_double()
        _check(load().dft_hartree_from_guess_dev(self.ctx, C.byref(g), _ptr(rho), _ptr(vh), tol, max_sweeps,
                                                 C.byref(sw), C.byref(ld)))
        return sw.value, ld.value

    def poisson_start(self, grid, net, rho, out, multigrid_cycles=0) -> dict:
        """Start values for the Jacobi solve into out (device): nested coarse grids, plus the
        network's correction (net not None), then up to multigrid_cycles V-cycles."""
        g = grid.c()
        info = dft_poisson_start_info()
        _check(load().dft_poisson_start_dev(self.ctx, C.byref(g), net.handle if net is not None else None, _ptr(rho),
                                            _ptr(out), int(multigrid_cycles), C.byref(info)))
        return {k: getattr(info, k) for k, _ in dft_poisson_start_info._fields_}

    def synthetic_density(self, grid, seed, out, kmin=1, kmax=8, wmin=0.3, wmax=2.0, ne_min=2, ne_max=40) -> int:
        g = grid.c()
        ne = C.c_int()
        _check(load().dft_synthetic_density_dev(self.ctx, C.byref(g), int(seed), kmin, kmax, wmin, wmax, ne_min,
                                                ne_max, _ptr(out), C.byref(ne)))
        return ne.value

    def hartree_energy(self, grid, rho, vh) -> float:
        g = grid.c()
        e = C.c_double()
        _check(load().dft_hartree_energy_dev(self.ctx, C.byref(g), _ptr(rho), _ptr(vh), C.byref(e)))
        return e.value

    def xc(self, grid, kind, na, nb, va=None, vb=None, energy=True):
        g = grid.c()
        e = C.c_double()
        _check(load().dft_xc_dev(self.ctx, C.byref(g), _kind(kind), _ptr(na), _ptr(nb), _ptr(va), _ptr(vb),
                                 C.byref(e) if energy else None))
        return e.value if energy else None

    def xc_evaluate(self, kind, m, na, nb, ga, gb, out5):
        _check(load().dft_xc_evaluate_dev(self.ctx, _kind(kind), m, _ptr(na), _ptr(nb), _ptr(ga), _ptr(gb),
                                          _ptr(out5)))

    def spin_density(self, npoints, psi, nbands, ld, occ, out):
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        _check(load().dft_spin_density_dev(self.ctx, npoints, _ptr(psi), nbands, ld, _dp(occ), _ptr(out)))

    def kinetic_energy(self, grid, psi, nbands, ld, occ) -> float:
        g = grid.c()
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        e = C.c_double()
        _check(load().dft_kinetic_energy_dev(self.ctx, C.byref(g), _ptr(psi), nbands, ld, _dp(occ), C.byref(e)))
        return e.value

    def nuclear_potential(self, grid, Z, xyz, vext):
        g = grid.c()
        Z = np.ascontiguousarray(Z, dtype=np.int32)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        _check(load().dft_nuclear_potential_dev(self.ctx, C.byref(g), len(Z), Z.ctypes.data_as(C.POINTER(C.c_int)),
                                                _dp(xyz), _ptr(vext)))

    def gram(self, grid, A, lda, ka, B, ldb, kb, precision=0) -> np.ndarray:
        g = grid.c()
        out = np.zeros((ka, kb))
        _check(load().dft_gram_dev(self.ctx, C.byref(g), _ptr(A), lda, ka, _ptr(B), ldb, kb, int(precision), _dp(out)))
        return out

    def screened_poisson(self, grid, src, x, q2, cycles=1):
        """x ~ (-lap_h + q2)^{-1} src by `cycles` multigrid cycles (the Kerker mixer's screening solve)."""
        g = grid.c()
        _check(load().dft_screened_poisson_dev(self.ctx, C.byref(g), _ptr(src), _ptr(x), float(q2), int(cycles)))

    def rotate(self, grid, V, ldv, k, Y, X, ldx, precision=0):
        """X = V * Y for band blocks (Y: k x m host matrix)."""
        g = grid.c()
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        _check(load().dft_rotate_dev(self.ctx, C.byref(g), _ptr(V), ldv, k, _dp(Y), Y.shape[1], _ptr(X), ldx,
                                     int(precision)))

    def solve_orbitals(self, grid, V, nocc, nbands, psi, ld, init=False, tol=1e-7, max_iterations=2000,
                       max_subspace=3, verbose=False, preconditioner=4, mixed_precision=0, preconditioner_net=None):
        g = grid.c()
        eig = np.zeros(nbands)
        o = dft_eig_opts(tol, max_iterations, max_subspace, int(verbose), int(preconditioner), int(mixed_precision),
                         preconditioner_net.handle if preconditioner_net is not None else None)
        it = C.c_int()
        _check(load().dft_solve_orbitals_dev(self.ctx, C.byref(g), _ptr(V), nocc, nbands, _ptr(psi), ld, int(init),
                                             _dp(eig), C.byref(o), C.byref(it)))
        return eig, it.value

    def scf_molecule(self, grid, molecule: Molecule, charge=None, multiplicity=1, functional=PZ81_KIND,
                     options: Optional[dft_scf_opts] = None, want_density=False, history=256):
        lib = load()
        g = grid.c()
        Z, xyz = molecule.arrays()
        charge = molecule.charge if charge is None else charge
        if options is None:
            options = default_scf_options()
        res = dft_scf_result()
        ne = int(Z.sum()) - charge
        eig = np.zeros(max(ne, 1) + 2)
        res.eigenvalues = _dp(eig)
        N = grid.getSize()
        da = db = None
        if want_density:
            da, db = np.zeros(N), np.zeros(N)
            res.alpha_density, res.beta_density = _dp(da), _dp(db)
        hist = (dft_scf_iteration * max(history, 1))()
        res.history = hist
        res.history_capacity = history
        _check(lib.dft_scf_molecule(self.ctx, C.byref(g), len(Z), Z.ctypes.data_as(C.POINTER(C.c_int)), _dp(xyz),
                                    charge, multiplicity, _kind(functional), C.byref(options), C.byref(res)))
        return SCFResult.from_c(res, eig, da, db, hist)

    def solve_atoms(self, Zs: Sequence[int], kinds: Sequence[int], points=2000, rmax=30.0):
        n = len(Zs)
        Za = np.ascontiguousarray(Zs, dtype=np.int32)
        Ka = np.ascontiguousarray([_kind(k) for k in kinds], dtype=np.int32)
        out = (dft_atom_result * n)()
        _check(load().dft_solve_atoms(self.ctx, n, Za.ctypes.data_as(C.POINTER(C.c_int)),
                                      Ka.ctypes.data_as(C.POINTER(C.c_int)), points, rmax, out))
        return [AtomResult.from_c(o) for o in out]


class PoissonNet:
    """The learned Poisson start's network (dft_pnet) on one engine."""

    def __init__(self, engine: "Engine", seed: int = 1, in_channels: int = 2):
        self.engine = engine
        h = C.c_void_p()
        _check(load().dft_pnet_create(engine.ctx, in_channels, int(seed), C.byref(h)))
        self.handle = h.value

    def close(self):
        if self.handle:
            load().dft_pnet_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def num_params(self) -> int:
        n = C.c_size_t()
        _check(load().dft_pnet_num_params(self.handle, C.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.num_params, dtype=np.float32)
        _check(load().dft_pnet_get_params(self.engine.ctx, self.handle, out.ctypes.data_as(C.POINTER(C.c_float)),
                                          out.size))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(load().dft_pnet_set_params(self.engine.ctx, self.handle, p.ctypes.data_as(C.POINTER(C.c_float)),
                                          p.size))

    def save(self, path: str) -> None:
        np.save(path, self.get_params())

    def load(self, path: str) -> None:
        self.set_params(np.load(path))

    def loss_grad(self, shape, x, t):
        """One forward/backward pass on a host volume: x (N, channels), t (N) -> (loss, grad, y)."""
        nx, ny, nz = shape
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        grad = np.zeros(self.num_params, dtype=np.float32)
        y = np.zeros(nx * ny * nz, dtype=np.float32)
        loss = C.c_double()
        fp = C.POINTER(C.c_float)
        _check(load().dft_pnet_loss_grad(self.engine.ctx, self.handle, nx, ny, nz, x.ctypes.data_as(fp),
                                         t.ctypes.data_as(fp), C.byref(loss), grad.ctypes.data_as(fp),
                                         y.ctypes.data_as(fp)))
        return loss.value, grad, y

    def train(self, grids, samples=256, validation=32, epochs=10, batch=4, lr=2e-3, lr_min=5e-5, seed=2026,
              target_tol=1e-10, target_max_sweeps=200000, kmin=1, kmax=8, wmin=0.3, wmax=2.0, ne_min=2, ne_max=40,
              smooth_sweeps=64, mse_weight=0.1, verbose=False) -> dict:
        o = dft_pnet_train_opts()
        o.samples, o.validation, o.epochs, o.batch = samples, validation, epochs, batch
        o.lr, o.lr_min, o.seed = lr, lr_min, seed
        o.target_tol, o.target_max_sweeps = target_tol, target_max_sweeps
        if not 1 <= len(grids) <= 4:
            raise ValueError("1 to 4 training grids")
        o.ngrids = len(grids)
        for i, g in enumerate(grids):
            o.grids[i] = g.c()
        o.kmin, o.kmax, o.wmin, o.wmax, o.ne_min, o.ne_max = kmin, kmax, wmin, wmax, ne_min, ne_max
        o.smooth_sweeps, o.mse_weight = smooth_sweeps, mse_weight
        o.verbose = int(verbose)
        r = dft_pnet_train_report()
        hist = (C.c_double * epochs)()
        r.epoch_loss = C.cast(hist, C.POINTER(C.c_double))
        r.epoch_loss_capacity = epochs
        _check(load().dft_pnet_train_poisson(self.engine.ctx, self.handle, C.byref(o), C.byref(r)))
        out = {k: getattr(r, k) for k, _ in dft_pnet_train_report._fields_ if k not in ("epoch_loss",
                                                                                      "epoch_loss_capacity")}
        out["epoch_loss"] = list(hist)
        return out

    def train_preconditioner(self, grid, V, nocc, nbands, samples=96, validation=16, epochs=12, batch=4, lr=2e-3,
                             lr_min=5e-5, seed=2026, cycles=12, verbose=False) -> dict:
        """Trains this network as the learned Davidson preconditioner (preconditioner -3) on the
        residual bands of a plain block eigensolve in the device potential V on `grid`; targets
        from `cycles` refined multigrid cycles.  Returns the training report."""
        o = dft_pnet_train_opts()
        o.samples, o.validation, o.epochs, o.batch = samples, validation, epochs, batch
        o.lr, o.lr_min, o.seed = lr, lr_min, seed
        o.target_tol, o.target_max_sweeps = 1e-7, cycles
        o.verbose = int(verbose)
        r = dft_pnet_train_report()
        hist = (C.c_double * epochs)()
        r.epoch_loss = C.cast(hist, C.POINTER(C.c_double))
        r.epoch_loss_capacity = epochs
        g = grid.c()
        _check(load().dft_pnet_train_preconditioner(self.engine.ctx, self.handle, C.byref(g), _ptr(V), int(nocc),
                                                    int(nbands), C.byref(o), C.byref(r)))
        out = {k: getattr(r, k) for k, _ in dft_pnet_train_report._fields_ if k not in ("epoch_loss",
                                                                                      "epoch_loss_capacity")}
        out["epoch_loss"] = list(hist)
        return out


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, DeviceArray):
        return x.ptr
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):  # a torch CUDA tensor
        return x.data_ptr()
    raise TypeError(f"expected a device buffer, got {type(x)}")


def default_scf_options(**kw) -> dft_scf_opts:
    o = dft_scf_opts()
    load().dft_scf_default_options(C.byref(o))
    scf_fields = {f for f, _ in dft_scf_opts._fields_}
    eig_fields = {f for f, _ in dft_eig_opts._fields_}
    for k, v in kw.items():
        if k == "poisson_net" and hasattr(v, "handle"):
            v = v.handle
        if k == "log_path" and isinstance(v, str):
            v = v.encode()
        if k not in scf_fields and not (k.startswith("eig_") and k[4:] in eig_fields):
            raise TypeError(f"unknown SCF option {k!r}")
        if k not in scf_fields:
            setattr(o.eig, k[4:], v)
        else:
            setattr(o, k, v)
    return o


# ----------------------------------------------------------------- results --------------
@dataclass
class EnergyComponents:
    """reference EnergyComponents (DFTData.h:47-54)."""
    kinetic: float = 0.0
    external: float = 0.0
    hartree: float = 0.0
    exchangeCorrelation: float = 0.0
    nuclearRepulsion: float = 0.0
    total: float = 0.0


@dataclass
class SCFResult:
    """reference SCFResult (DFTData.h:56-79) / MolecularResult (:86-91)."""
    energy: EnergyComponents
    iterations: int
    converged: bool
    densityDifference: float
    energyDifference: float
    maxKSResidual: float
    eigenvalues: List[float]
    alphaDensity: Optional[np.ndarray] = None
    betaDensity: Optional[np.ndarray] = None
    history: list = field(default_factory=list)
    seconds: float = 0.0
    n_alpha: int = 0
    n_beta: int = 0
    convergence: dict = field(default_factory=dict)

    @property
    def total(self):
        return self.energy.total

    @classmethod
    def from_c(cls, r: dft_scf_result, eig, da, db, hist):
        e = EnergyComponents(r.kinetic, r.external, r.hartree, r.exchange_correlation, r.nuclear_repulsion, r.total)
        h = [{k: getattr(hist[i], k) for k, _ in dft_scf_iteration._fields_} for i in range(r.history_len)]
        conv = {"lastEnergyCriterionIteration": r.last_energy_criterion_iteration,
                "lastDensityCriterionIteration": r.last_density_criterion_iteration,
                "lastKSCriterionIteration": r.last_ks_criterion_iteration,
                "finalEnergyDifference": r.energy_difference, "finalDensityDifference": r.density_difference,
                "finalKSResidual": r.max_ks_residual, "finalMixing": r.final_mixing,
                "minimumEnergyDifference": r.min_energy_difference,
                "minimumDensityDifference": r.min_density_difference, "minimumKSResidual": r.min_ks_residual}
        return cls(e, r.iterations, bool(r.converged), r.density_difference, r.energy_difference, r.max_ks_residual,
                   list(eig[: r.n_alpha + r.n_beta]), da, db, h, r.seconds, r.n_alpha, r.n_beta, conv)

    def to_dict(self, charge: int = 0) -> dict:
        """The reference's MolecularResult (DFTData.h:86-91) without the grid fields, plus the
        convergence analysis (MolecularSCFHelpers.h:47-72) and the phase times summed over the
        iterations (seconds, the MolecularSCFTiming fields this engine measures)."""
        phases = {k: 1e-3 * sum(h[k] for h in self.history)
                  for k in ("ms_hartree", "ms_xc", "ms_orbitals", "ms_density", "ms_energy", "ms_total")}
        timing = {"hartree": phases["ms_hartree"], "exchangeCorrelation": phases["ms_xc"],
                  "orbitals": phases["ms_orbitals"], "outputDensity": phases["ms_density"],
                  "totalEnergy": phases["ms_energy"], "totalIterations": phases["ms_total"], "total": self.seconds}
        return {"electrons": self.n_alpha + self.n_beta, "charge": charge,
                "scf": {"energy": vars(self.energy), "iterations": self.iterations, "converged": self.converged,
                        "densityDifference": self.densityDifference, "energyDifference": self.energyDifference,
                        "maxKSResidual": self.maxKSResidual,
                        "alphaEigenvalues": self.eigenvalues[: self.n_alpha],
                        "betaEigenvalues": self.eigenvalues[self.n_alpha:]},
                "convergenceAnalysis": self.convergence, "timing": timing, "history": self.history}

    def write_json(self, path: str, charge: int = 0) -> None:
        """The result file: one JSON document (to_dict)."""
        import json
        with open(path, "w") as f:
            json.dump(self.to_dict(charge), f, indent=1)


@dataclass
class AtomResult:
    """reference AtomicResult (DFTData.h:81-84) for one radial run."""
    Z: int
    kind: int
    energy: EnergyComponents
    iterations: int
    converged: bool
    densityDifference: float
    maxKSResidual: float
    eigenvalues: List[float]
    status: int

    @classmethod
    def from_c(cls, o: dft_atom_result):
        e = EnergyComponents(o.kinetic, o.external, o.hartree, o.exchange_correlation, 0.0, o.total)
        return cls(o.Z, o.kind, e, o.iterations, bool(o.converged), o.density_difference, o.max_ks_residual,
                   list(o.eigenvalues[: o.n_orbitals]), o.status)


# ----------------------------------------------------------------- reference-named API --
_default_engine: Optional[Engine] = None


def engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine(0)
    return _default_engine


def applyMolecularKohnShamHamiltonian(grid: CartesianGrid, effectivePotential, psi) -> np.ndarray:
    """reference KohnShamHamiltonianMolecule.h:7-11 (host vectors in, new host vector out)."""
    e = engine()
    N = grid.getSize()
    V, P = e.upload(effectivePotential), e.upload(psi)
    if V.n != N or P.n != N:
        raise ValueError("La funcion de onda y la malla cartesiana deben tener el mismo tamano.")
    H = e.array(N)
    e.apply_hamiltonian(grid, V, P, H, 1, N)
    return H.to_host()


def calculateHartreePotential(grid: CartesianGrid, density) -> np.ndarray:
    """reference HartreePotentialMolecule.h:7-10."""
    e = engine()
    rho = e.upload(density)
    if rho.n != grid.getSize():
        raise ValueError("La densidad molecular y la malla cartesiana deben tener el mismo tamano.")
    vh = e.array(rho.n)
    e.hartree(grid, rho, vh)
    return vh.to_host()


def calculateHartreeEnergy(grid: CartesianGrid, density, hartreePotential) -> float:
    e = engine()
    return e.hartree_energy(grid, e.upload(density), e.upload(hartreePotential))


def calculateMolecularSpinExchangeCorrelationPotential(functional, grid, alphaDensity, betaDensity, spin: int):
    """reference ExchangeCorrelationMolecule.h:8-14."""
    if spin not in (0, 1):
        raise ValueError("El canal de spin debe ser 0 (alpha) o 1 (beta).")
    e = engine()
    na, nb = e.upload(alphaDensity), e.upload(betaDensity)
    v = e.array(na.n)
    e.xc(grid, functional, na, nb, v if spin == 0 else None, v if spin == 1 else None, energy=False)
    return v.to_host()


def calculateMolecularExchangeCorrelationEnergy(functional, grid, alphaDensity, betaDensity) -> float:
    """reference ExchangeCorrelationMolecule.h:16-21."""
    e = engine()
    return e.xc(grid, functional, e.upload(alphaDensity), e.upload(betaDensity), None, None, energy=True)


@dataclass
class MolecularOrbital:
    """reference MolecularOrbital (DFTData.h:34-39)."""
    spin: int
    electrons: int
    eigenvalue: float
    psi: np.ndarray


def solveMolecularOrbitals(grid, effectivePotential, numberOfOrbitals: int, occupations, spin=0,
                           initialOrbitals: Sequence[MolecularOrbital] = (), extra_bands: int = 3,
                           tol: float = 1e-7):
    """reference EigenvalueSolverMolecule.h:20-28 (block Davidson on the GPU)."""
    if numberOfOrbitals <= 0:
        raise ValueError("El numero de orbitales debe ser mayor que cero.")
    if len(occupations) != numberOfOrbitals:
        raise ValueError("Las ocupaciones no coinciden con el numero de orbitales.")
    e = engine()
    N = grid.getSize()
    nb = min(numberOfOrbitals + extra_bands, N)
    V = e.upload(effectivePotential)
    init = len(initialOrbitals) > 0
    block = np.zeros((nb, N))
    if init:
        for i, o in enumerate(initialOrbitals[:nb]):
            block[i] = o.psi
    psi = e.upload(block)
    eig, _ = e.solve_orbitals(grid, V, numberOfOrbitals, nb, psi, N, init=init, tol=tol)
    P = psi.to_host((nb, N))
    return [MolecularOrbital(spin, int(occupations[i]), float(eig[i]), P[i].copy()) for i in range(numberOfOrbitals)]


def solveMolecularSelfConsistentField(grid: CartesianGrid, molecule: Molecule, charge: int, multiplicity: int,
                                      functional, options: Optional[dft_scf_opts] = None,
                                      want_density: bool = False) -> SCFResult:
    """reference SelfConsistentFieldMolecule.h:8-14."""
    return engine().scf_molecule(grid, molecule, charge, multiplicity, functional, options, want_density)


def solveAtom(grid: RadialGrid, Z: int, functional) -> AtomResult:
    """reference AtomicDFT.h:7-11 with getAtomicConfiguration(Z)."""
    return engine().solve_atoms([Z], [_kind(functional)], grid.points, grid.rmax)[0]


def solveAtoms(grid: RadialGrid, Zs: Sequence[int], functionals: Sequence) -> List[AtomResult]:
    """Many independent solveAtom runs in one persistent launch."""
    return engine().solve_atoms(list(Zs), [_kind(f) for f in functionals], grid.points, grid.rmax)
