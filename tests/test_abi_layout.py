"""CPU: the ctypes structures in dft_b200/__init__.py match include/dft_b200.h field by field
(size and offset of every member, compiled with the system C compiler), and the Python option
helpers reject names that the C structures do not have."""
import ctypes as C
import os
import subprocess

import pytest

import dft_b200 as d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "dft_grid": d.dft_grid,
    "dft_eig_opts": d.dft_eig_opts,
    "dft_scf_opts": d.dft_scf_opts,
    "dft_scf_iteration": d.dft_scf_iteration,
    "dft_scf_result": d.dft_scf_result,
    "dft_atom_result": d.dft_atom_result,
    "dft_poisson_start_info": d.dft_poisson_start_info,
    "dft_pnet_train_opts": d.dft_pnet_train_opts,
    "dft_pnet_train_report": d.dft_pnet_train_report,
    "dft_autotune_report": d.dft_autotune_report,
}


def _c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dft_b200.h"', "int main(void) {"]
    for name, cls in STRUCTS.items():
        lines.append(f'printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        s, f, v = line.split()
        table[(s, f)] = int(v)
    return table


def test_ctypes_structs_match_header(tmp_path):
    table = _c_layout(tmp_path)
    for name, cls in STRUCTS.items():
        assert C.sizeof(cls) == table[(name, "sizeof")], name
        for field, _ in cls._fields_:
            assert getattr(cls, field).offset == table[(name, field)], (name, field)


def test_scf_option_names_are_checked():
    o = d.default_scf_options(mixer=1, adaptive_eig_tol=1, eig_preconditioner=-2, smearing_kt=0.01,
                              poisson_start=d.POISSON_MULTIGRID)
    assert (o.mixer, o.adaptive_eig_tol, o.eig.preconditioner, o.poisson_start) == (1, 1, -2, d.POISSON_MULTIGRID)
    assert o.smearing_kt == 0.01
    for bad in ("eig_tol_adaptive", "mixing", "eig_nonexistent"):
        with pytest.raises(TypeError):
            d.default_scf_options(**{bad: 1})


def test_defaults_keep_the_reference_method():
    o = d.default_scf_options()
    assert o.poisson_start == d.POISSON_COLD and o.mixer == 0 and o.adaptive_eig_tol == 0
    assert o.smearing_kt == 0.0 and o.eig.mixed_precision == 0 and not o.poisson_net
