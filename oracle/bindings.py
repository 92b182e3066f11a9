"""ctypes bindings for the two CPU checkers (test infrastructure only).

``Port``  -> oracle/liboracle.so, the plain-C restatement in dft_oracle.c.
``Ref``   -> oracle/_ref/libdft_ref.so, the reference sources compiled by
            oracle/Makefile (present only where the reference tree was available
            at build time).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of bench.py use
this module, and only as the checker.  Grids are passed as ``n=(nx,ny,nz)`` and
``bounds=(xmin,xmax,ymin,ymax,zmin,zmax)`` exactly like ``CartesianGrid``
(reference CartesianGrid.cpp:5-48).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdft_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)

PZ81, PBE96 = 0, 1


def _d(a):
    return a.ctypes.data_as(_dp)


def _arr(x, dtype=np.float64):
    return np.ascontiguousarray(np.asarray(x, dtype=dtype))


def build_port() -> str:
    """Compile liboracle.so with the committed Makefile if it is missing or stale."""
    src = os.path.join(HERE, "dft_oracle.c")
    if (not os.path.exists(PORT_SO)) or os.path.getmtime(PORT_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return PORT_SO


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class _Lib:
    def __init__(self, path, prefix):
        self.lib = C.CDLL(path)
        self.p = prefix

    def fn(self, name):
        return getattr(self.lib, self.p + name)

    def check(self, rc):
        if rc != 0:
            msg = self.fn("last_error")
            msg.restype = C.c_char_p
            raise RuntimeError(msg().decode(errors="replace"))

    # ---- 3D operators -------------------------------------------------------
    def grid_args(self, n, bounds):
        na = np.asarray(n, dtype=np.int64)
        ba = _arr(bounds)
        return na, ba

    def apply_hamiltonian(self, n, bounds, V, psi):
        na, ba = self.grid_args(n, bounds)
        V, psi = _arr(V), _arr(psi)
        out = np.empty_like(psi)
        self.check(self.fn("apply_hamiltonian")(na.ctypes.data_as(_lp), _d(ba), _d(V), _d(psi), _d(out)))
        return out

    def hartree_potential(self, n, bounds, rho):
        na, ba = self.grid_args(n, bounds)
        rho = _arr(rho)
        out = np.empty_like(rho)
        self.check(self.fn("hartree_potential")(na.ctypes.data_as(_lp), _d(ba), _d(rho), _d(out)))
        return out

    def hartree_energy(self, n, bounds, rho, vh):
        na, ba = self.grid_args(n, bounds)
        rho, vh = _arr(rho), _arr(vh)
        e = C.c_double()
        self.check(self.fn("hartree_energy")(na.ctypes.data_as(_lp), _d(ba), _d(rho), _d(vh), C.byref(e)))
        return e.value

    def xc_evaluate(self, kind, na, nb, ga, gb):
        na, nb, ga, gb = map(_arr, (na, nb, ga, gb))
        out = np.empty((na.size, 5))
        self.check(self.fn("xc_evaluate")(kind, C.c_long(na.size), _d(na), _d(nb), _d(ga), _d(gb), _d(out)))
        return out

    def xc_potential(self, kind, n, bounds, na, nb, spin):
        nn, ba = self.grid_args(n, bounds)
        na, nb = _arr(na), _arr(nb)
        out = np.empty_like(na)
        self.check(self.fn("xc_potential")(kind, nn.ctypes.data_as(_lp), _d(ba), _d(na), _d(nb), spin, _d(out)))
        return out

    def xc_energy(self, kind, n, bounds, na, nb):
        nn, ba = self.grid_args(n, bounds)
        na, nb = _arr(na), _arr(nb)
        e = C.c_double()
        self.check(self.fn("xc_energy")(kind, nn.ctypes.data_as(_lp), _d(ba), _d(na), _d(nb), C.byref(e)))
        return e.value

    def nuclear_potential(self, n, bounds, Z, xyz):
        nn, ba = self.grid_args(n, bounds)
        Z = _arr(Z, np.int32)
        xyz = _arr(xyz)
        out = np.empty(int(np.prod(n)))
        self.check(self.fn("nuclear_potential")(nn.ctypes.data_as(_lp), _d(ba), len(Z), Z.ctypes.data_as(_ip),
                                                _d(xyz), _d(out)))
        return out

    def nuclear_repulsion(self, Z, xyz):
        Z = _arr(Z, np.int32)
        xyz = _arr(xyz)
        e = C.c_double()
        self.check(self.fn("nuclear_repulsion")(len(Z), Z.ctypes.data_as(_ip), _d(xyz), C.byref(e)))
        return e.value

    def kinetic_energy(self, n, bounds, psi, electrons):
        nn, ba = self.grid_args(n, bounds)
        psi = _arr(psi)
        el = _arr(electrons, np.int32)
        e = C.c_double()
        self.check(self.fn("kinetic_energy")(nn.ctypes.data_as(_lp), _d(ba), len(el), _d(psi),
                                             el.ctypes.data_as(_ip), C.byref(e)))
        return e.value

    def spin_density(self, psi, electrons):
        psi = _arr(psi)
        el = _arr(electrons, np.int32)
        N = psi.shape[-1]
        out = np.empty(N)
        self.check(self.fn("spin_density")(C.c_long(N), len(el), _d(psi), el.ctypes.data_as(_ip), _d(out)))
        return out

    def solve_orbitals(self, n, bounds, V, norb, init=None):
        nn, ba = self.grid_args(n, bounds)
        V = _arr(V)
        N = V.size
        psi = np.empty((norb, N))
        eig = np.empty(norb)
        ip = _d(_arr(init)) if init is not None else None
        keep = _arr(init) if init is not None else None
        if keep is not None:
            ip = _d(keep)
        self.check(self.fn("solve_orbitals")(nn.ctypes.data_as(_lp), _d(ba), _d(V), norb, ip, _d(psi), _d(eig)))
        return eig, psi

    def scf_molecule(self, n, bounds, Z, xyz, charge, multiplicity, kind, want_density=False):
        nn, ba = self.grid_args(n, bounds)
        Z = _arr(Z, np.int32)
        xyz = _arr(xyz)
        e6 = np.zeros(6)
        st = np.zeros(4)
        eig = np.zeros(512)
        N = int(np.prod(n))
        dens = np.zeros(2 * N) if want_density else None
        self.check(self.fn("scf_molecule")(nn.ctypes.data_as(_lp), _d(ba), len(Z), Z.ctypes.data_as(_ip), _d(xyz),
                                           charge, multiplicity, kind, _d(e6), _d(st), 512, _d(eig),
                                           _d(dens) if dens is not None else None))
        ne = int(sum(Z)) - charge
        return {
            "kinetic": e6[0], "external": e6[1], "hartree": e6[2], "xc": e6[3], "nuclear": e6[4], "total": e6[5],
            "iterations": int(st[0]), "converged": bool(st[1]), "dRho": st[2], "KS": st[3],
            "eigenvalues": eig[:ne].tolist(),
            "density": dens,
        }

    def scf_sample(self, n, bounds, Z, xyz, multiplicity, kind, iterations=1):
        """Seconds for (initial densities, mean SCF iteration) of the reference algorithm."""
        nn, ba = self.grid_args(n, bounds)
        Z = _arr(Z, np.int32)
        xyz = _arr(xyz)
        s = np.zeros(2)
        self.check(self.fn("scf_sample")(nn.ctypes.data_as(_lp), _d(ba), len(Z), Z.ctypes.data_as(_ip), _d(xyz),
                                         multiplicity, kind, iterations, _d(s)))
        return float(s[0]), float(s[1])

    def scf_to_de(self, n, bounds, Z, xyz, multiplicity, kind, de_stop=1e-6, max_iterations=250):
        """The reference's SCF loop to |dE| < de_stop: (seconds, init seconds, iterations,
        energy, last |dE|).  Reference library only (ref_scf_to_de)."""
        nn, ba = self.grid_args(n, bounds)
        Z = _arr(Z, np.int32)
        xyz = _arr(xyz)
        out = np.zeros(5)
        self.check(self.fn("scf_to_de")(nn.ctypes.data_as(_lp), _d(ba), len(Z), Z.ctypes.data_as(_ip), _d(xyz),
                                        multiplicity, kind, C.c_double(de_stop), max_iterations, _d(out)))
        return float(out[0]), float(out[1]), int(out[2]), float(out[3]), float(out[4])

    # ---- radial -------------------------------------------------------------
    def solve_atom(self, Z, kind, points=2000, rmax=30.0):
        e5 = np.zeros(5)
        st = np.zeros(4)
        eig = np.zeros(32)
        nw = C.c_int()
        self.check(self.fn("solve_atom")(Z, kind, C.c_long(points), C.c_double(rmax), _d(e5), _d(st), 32, _d(eig),
                                         C.byref(nw)))
        return {"kinetic": e5[0], "external": e5[1], "hartree": e5[2], "xc": e5[3], "total": e5[4],
                "iterations": int(st[0]), "converged": bool(st[1]), "dRho": st[2], "KS": st[3],
                "eigenvalues": eig[: nw.value].tolist()}

    def radial_hartree(self, points, rmax, rho):
        rho = _arr(rho)
        out = np.empty_like(rho)
        self.check(self.fn("radial_hartree")(C.c_long(points), C.c_double(rmax), _d(rho), _d(out)))
        return out

    def radial_xc_potential(self, kind, points, rmax, na, nb, spin):
        na, nb = _arr(na), _arr(nb)
        out = np.empty_like(na)
        self.check(self.fn("radial_xc_potential")(kind, C.c_long(points), C.c_double(rmax), _d(na), _d(nb), spin,
                                                  _d(out)))
        return out

    def radial_xc_energy(self, kind, points, rmax, na, nb):
        na, nb = _arr(na), _arr(nb)
        e = C.c_double()
        self.check(self.fn("radial_xc_energy")(kind, C.c_long(points), C.c_double(rmax), _d(na), _d(nb),
                                               C.byref(e)))
        return e.value

    def radial_solve_orbital(self, points, rmax, veff, l, index):
        veff = _arr(veff)
        eig = C.c_double()
        u = np.empty(points)
        self.check(self.fn("radial_solve_orbital")(C.c_long(points), C.c_double(rmax), _d(veff), l, index,
                                                   C.byref(eig), _d(u)))
        return eig.value, u

    def radial_sturm_count(self, points, rmax, veff, l, energy):
        veff = _arr(veff)
        c = C.c_long()
        self.check(self.fn("radial_sturm_count")(C.c_long(points), C.c_double(rmax), _d(veff), l,
                                                 C.c_double(energy), C.byref(c)))
        return c.value

    def atomic_configuration(self, Z):
        rows = np.zeros(4 * 16, dtype=np.int32)
        nr = C.c_int()
        self.check(self.fn("atomic_configuration")(Z, 16, rows.ctypes.data_as(_ip), C.byref(nr)))
        return rows[: 4 * nr.value].reshape(-1, 4).tolist()


class Port(_Lib):
    """The plain-C restatement (oracle/dft_oracle.c)."""

    def __init__(self):
        super().__init__(build_port(), "oracle_")


class Ref(_Lib):
    """The reference sources compiled into oracle/_ref/libdft_ref.so."""

    def __init__(self):
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        super().__init__(REF_SO, "ref_")
