"""CPU: the C usage shown for integrators compiles against include/dft_b200.h (syntax and
types only; nothing runs without a GPU)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

EXAMPLE = r"""
#include <stdio.h>
#include "dft_b200.h"

int main(void) {
    dft_context* ctx;
    if (dft_context_create(0, &ctx) != DFT_OK) { fprintf(stderr, "%s\n", dft_last_error_message()); return 1; }
    dft_grid g = {48, 48, 48, -7.05, 7.05, -7.05, 7.05, -7.05, 7.05};
    int Z[2] = {1, 1};
    double xyz[6] = {-0.7, 0, 0, 0.7, 0, 0};
    dft_scf_opts o;
    dft_scf_default_options(&o);
    o.poisson_start = DFT_POISSON_MULTIGRID;
    o.eig.mixed_precision = 1;
    o.eig.preconditioner = -2;
    o.mixer = 1;
    o.adaptive_eig_tol = 1;
    dft_pnet* net;
    dft_pnet_create(ctx, 2, 7, &net);
    dft_pnet_train_opts t = {0};
    t.samples = 48; t.validation = 8; t.epochs = 10; t.batch = 4; t.lr = 3e-3; t.lr_min = 1e-4;
    t.target_tol = 1e-10; t.target_max_sweeps = 200000; t.ngrids = 1; t.grids[0] = g;
    t.kmin = 1; t.kmax = 8; t.wmin = 0.3; t.wmax = 2.0; t.ne_min = 2; t.ne_max = 40;
    dft_pnet_train_report rep = {0};
    dft_pnet_train_poisson(ctx, net, &t, &rep);
    o.poisson_net = net;
    dft_scf_result r = {0};
    if (dft_scf_molecule(ctx, &g, 2, Z, xyz, 0, 1, DFT_XC_PZ81, &o, &r) != DFT_OK)
        fprintf(stderr, "%s\n", dft_last_error_message());
    printf("E = %.10f after %d iterations\n", r.total, r.iterations);
    dft_pnet_destroy(net);
    dft_context_destroy(ctx);
    return 0;
}
"""


def test_documented_c_usage_compiles(tmp_path):
    src = tmp_path / "example.c"
    src.write_text(EXAMPLE)
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    str(src)], check=True)


def test_documented_cpp_shim_compiles_standalone(tmp_path):
    """The C++ layer's C ABI part is valid C++ too (the shim includes it from C++)."""
    src = tmp_path / "example.cpp"
    src.write_text(EXAMPLE)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    str(src)], check=True)
