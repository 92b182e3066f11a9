// extern "C" boundary of libdft_b200 (declared in include/dft_b200.h): argument checks,
// context and workspace management, and the translation of dftb::Error into status codes.
#include <cstring>
#include <string>

#include "neural.h"
#include "ops.h"

namespace {

thread_local std::string g_error;

template <class F>
dft_status_t guard(dft_context* ctx, F&& f) {
    try {
        if (ctx) {
            cudaError_t e = cudaSetDevice(ctx->device);
            if (e != cudaSuccess) {
                g_error = std::string("cudaSetDevice failed: ") + cudaGetErrorString(e);
                return DFT_CUDA_ERROR;
            }
        }
        f();
        return DFT_OK;
    } catch (const dftb::Error& e) {
        g_error = e.what();
        return e.status;
    } catch (const std::exception& e) {
        g_error = e.what();
        return DFT_INVALID_ARGUMENT;
    }
}

#define NEED(cond, msg)                                               \
    do {                                                              \
        if (!(cond)) ::dftb::fail(DFT_INVALID_ARGUMENT, "%s", msg);   \
    } while (0)

}  // namespace

namespace dftb {

void* ws_get(dft_context* ctx, int slot, size_t bytes) {
    static_assert(WS_NUM <= (int)(sizeof(ctx->ws) / sizeof(ctx->ws[0])), "workspace slots");
    if (slot < 0 || slot >= WS_NUM) fail(DFT_INVALID_ARGUMENT, "workspace slot %d out of range", slot);
    Workspace& w = ctx->ws[slot];
    if (w.bytes >= bytes && w.ptr) return w.ptr;
    if (w.ptr) {
        // kernels queued on the stream may still read the old buffer
        DFT_CUDA(cudaStreamSynchronize(ctx->stream));
        DFT_CUDA(cudaFree(w.ptr));
        w.ptr = nullptr;
        w.bytes = 0;
    }
    const size_t want = std::max<size_t>(bytes, 256);
    DFT_CUDA(cudaMalloc(&w.ptr, want));
    w.bytes = want;
    return w.ptr;
}

double* pinned(dft_context* ctx, size_t count) {
    const size_t bytes = std::max<size_t>(count, 8) * sizeof(double);
    if (ctx->host_pinned_bytes < bytes) {
        DFT_CUDA(cudaStreamSynchronize(ctx->stream));
        if (ctx->host_pinned) DFT_CUDA(cudaFreeHost(ctx->host_pinned));
        ctx->host_pinned = nullptr;
        DFT_CUDA(cudaMallocHost(&ctx->host_pinned, bytes));
        ctx->host_pinned_bytes = bytes;
    }
    return ctx->host_pinned;
}

void sync(dft_context* ctx) { DFT_CUDA(cudaStreamSynchronize(ctx->stream)); }

}  // namespace dftb

extern "C" {

const char* dft_last_error_message(void) { return g_error.c_str(); }
const char* dft_version(void) { return "dft_b200 0.1 (sm_100a)"; }

dft_status_t dft_context_create(int device, dft_context** out) {
    return guard(nullptr, [&] {
        NEED(out, "out is NULL");
        int n = 0;
        DFT_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) dftb::fail(DFT_INVALID_ARGUMENT, "device %d out of range (%d devices)", device, n);
        DFT_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        DFT_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major < 10)
            dftb::fail(DFT_CUDA_ERROR, "device %d is sm_%d%d; the library is compiled for sm_100a", device, prop.major, prop.minor);
        // the allocation-free Hartree entry point's fixed array: load its module now, while
        // allocating is allowed, rather than at that entry point's first call
        dftb::noalloc_scratch(device);
        auto* c = new dft_context();
        c->device = device;
        c->num_sms = prop.multiProcessorCount;
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete c;
            dftb::fail(DFT_CUDA_ERROR, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
        }
        *out = c;
    });
}

dft_status_t dft_context_destroy(dft_context* ctx) {
    if (!ctx) return DFT_OK;
    dft_status_t s = guard(ctx, [&] {
        DFT_CUDA(cudaStreamSynchronize(ctx->stream));
        for (auto& w : ctx->ws)
            if (w.ptr) cudaFree(w.ptr);
        if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
        if (ctx->gram_ticket) cudaFree(ctx->gram_ticket);
        if (ctx->dev_status) cudaFree(ctx->dev_status);
        for (auto& kv : ctx->buf_pool) cudaFree(kv.second);
        ctx->buf_pool.clear();
        for (auto& kv : ctx->radial_tables) cudaFree(kv.second.dens);
        for (auto& kv : ctx->mg_graphs) cudaGraphExecDestroy(kv.second.exec);
        cudaStreamDestroy(ctx->stream);
    });
    delete ctx;
    return s;
}

dft_status_t dft_context_synchronize(dft_context* ctx) {
    return guard(ctx, [&] {
        NEED(ctx, "context is NULL");
        dftb::sync(ctx);
        dftb::check_device_status(ctx, "a kernel on the context's stream");
    });
}

dft_status_t dft_context_set_tuning(dft_context* ctx, const char* key, long value) {
    return guard(ctx, [&] {
        NEED(ctx && key, "NULL argument");
        const std::string k(key);
        if (k == "jacobi_sweeps_per_launch") {
            NEED(value == 0 || value == -2 || value == -1 || value == 1 || value == 2 || value == 4 || value == 8,
                 "jacobi_sweeps_per_launch must be 0 (auto), -2 (cluster), -1 (persistent), 1, 2, 4 or 8");
            ctx->jacobi_sweeps_per_launch = (int)value;
        } else if (k == "network_tensor_cores") {
            NEED(value == 0 || value == 1, "network_tensor_cores must be 0 or 1");
            ctx->net_tensor_cores = (int)value;
        } else if (k == "grid_barrier_poll_limit") {
            NEED(value >= 0, "grid_barrier_poll_limit must be >= 0 (0 = default)");
            ctx->grid_barrier_poll_limit = value;
        } else if (k == "radial_pivot_exponent") {
            NEED(value >= -300 && value <= 300, "radial_pivot_exponent must be in [-300, 300]");
            ctx->radial_pivot_exp = (int)value;
        } else if (k == "multigrid_graphs") {
            NEED(value == 0 || value == 1, "multigrid_graphs must be 0 or 1");
            ctx->multigrid_graphs = (int)value;
        } else if (k == "tensor_core_ring") {
            NEED(value == 0 || value == 1, "tensor_core_ring must be 0 or 1");
            ctx->tc_ring = (int)value;
        } else if (k == "hpsi_variant") {
            NEED(value >= 0 && value <= 3, "hpsi_variant must be 0, 1, 2 or 3");
            ctx->hpsi_variant = (int)value;
        } else if (k == "multigrid_fused_restriction" || k == "multigrid_coarsest_sor") {
            NEED(value == 0 || value == 1, "multigrid keys take 0 or 1");
            (k == "multigrid_fused_restriction" ? ctx->mg_fused_restrict : ctx->mg_coarsest_sor) = (int)value;
            // captured multigrid cycles hold the old launch sequence
            dftb::sync(ctx);
            for (auto& kv : ctx->mg_graphs) cudaGraphExecDestroy(kv.second.exec);
            ctx->mg_graphs.clear();
        } else if (k == "hpsi_zchunk") {
            NEED(value >= 0 && value <= 65536, "hpsi_zchunk must be 0 (auto) or a plane count");
            ctx->hpsi_zchunk = (int)value;
        } else if (k == "tensor_core_tma") {
            NEED(value == 0 || value == 1, "tensor_core_tma must be 0 or 1");
            ctx->tc_tma = (int)value;
        } else if (k == "orthonormalise_adaptive") {
            NEED(value == 0 || value == 1, "orthonormalise_adaptive must be 0 or 1");
            ctx->ortho_adaptive = (int)value;
        } else if (k == "hpsi_bands_per_thread") {
            NEED(value == 0 || value == 1 || value == 2 || value == 4 || value == 8,
                 "hpsi_bands_per_thread must be 0 (auto), 1, 2, 4 or 8");
            ctx->hpsi_bands_per_thread = (int)value;
        } else {
            dftb::fail(DFT_INVALID_ARGUMENT, "unknown tuning key '%s'", key);
        }
    });
}

dft_status_t dft_autotune(dft_context* ctx, const dft_grid* g, int nbands, dft_autotune_report* report) {
    return guard(ctx, [&] {
        NEED(ctx && g, "NULL argument");
        dftb::autotune(ctx, dftb::make_grid(g), nbands, report);
    });
}

void* dft_context_stream(dft_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
long long dft_context_launch_count(dft_context* ctx) { return ctx ? ctx->launches : 0; }

long long dft_context_counter(dft_context* ctx, const char* name) {
    if (!ctx || !name) return -1;
    if (!std::strcmp(name, "launches")) return ctx->launches;
    if (!std::strcmp(name, "tensor_core_products")) return ctx->tc_launches;
    return -1;
}

dft_status_t dft_device_alloc(dft_context* ctx, size_t bytes, void** out) {
    return guard(ctx, [&] {
        NEED(ctx && out, "NULL argument");
        DFT_CUDA(cudaMalloc(out, std::max<size_t>(bytes, 1)));
    });
}
dft_status_t dft_device_free(dft_context* ctx, void* ptr) {
    return guard(ctx, [&] {
        NEED(ctx, "context is NULL");
        if (ptr) {
            DFT_CUDA(cudaStreamSynchronize(ctx->stream));
            DFT_CUDA(cudaFree(ptr));
        }
    });
}
dft_status_t dft_copy_h2d(dft_context* ctx, void* dst, const void* src, size_t bytes) {
    return guard(ctx, [&] {
        NEED(ctx && dst && src, "NULL argument");
        DFT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        dftb::sync(ctx);
    });
}
dft_status_t dft_copy_d2h(dft_context* ctx, void* dst, const void* src, size_t bytes) {
    return guard(ctx, [&] {
        NEED(ctx && dst && src, "NULL argument");
        DFT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        dftb::sync(ctx);
    });
}

dft_status_t dft_apply_hamiltonian_dev(dft_context* ctx, const dft_grid* g, const double* V, const double* psi,
                                       double* hpsi, int nbands, long ld) {
    return guard(ctx, [&] {
        NEED(ctx && V && psi && hpsi, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        NEED(nbands >= 0, "nbands must be >= 0");
        NEED(ld >= G.N, "ld must be >= nx*ny*nz");
        dftb::apply_hamiltonian(ctx, G, V, psi, hpsi, nbands, ld);
    });
}

dft_status_t dft_hartree_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh, double tol,
                             long max_sweeps, long* sweeps_out, double* last_diff_out) {
    return guard(ctx, [&] {
        NEED(ctx && rho && vh, "NULL argument");
        NEED(rho != vh, "rho and vh must not alias");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::JacobiResult r = dftb::hartree(ctx, G, rho, vh, tol, max_sweeps);
        dftb::sync(ctx);
        if (sweeps_out) *sweeps_out = r.sweeps;
        if (last_diff_out) *last_diff_out = r.last_diff;
    });
}

dft_status_t dft_hartree_from_guess_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh,
                                        double tol, long max_sweeps, long* sweeps_out, double* last_diff_out) {
    return guard(ctx, [&] {
        NEED(ctx && rho && vh, "NULL argument");
        NEED(rho != vh, "rho and vh must not alias");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::JacobiResult r = dftb::hartree(ctx, G, rho, vh, tol, max_sweeps, vh);
        dftb::sync(ctx);
        if (sweeps_out) *sweeps_out = r.sweeps;
        if (last_diff_out) *last_diff_out = r.last_diff;
    });
}

dft_status_t dft_hartree_noalloc_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh, double tol,
                                     long max_sweeps, long* sweeps_out, double* last_diff_out) {
    return guard(ctx, [&] {
        NEED(ctx && rho && vh, "NULL argument");
        NEED(rho != vh, "rho and vh must not alias");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::JacobiResult r = dftb::hartree_noalloc(ctx, G, rho, vh, tol, max_sweeps);
        if (sweeps_out) *sweeps_out = r.sweeps;
        if (last_diff_out) *last_diff_out = r.last_diff;
    });
}

dft_status_t dft_zslab_jacobi_init_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, double Q,
                                       const double* guess, double* v) {
    return guard(ctx, [&] {
        NEED(ctx && v, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::zslab_jacobi_init(ctx, G, z_lo, z_hi, Q, guess, v);
        dftb::sync(ctx);
    });
}

dft_status_t dft_zslab_jacobi_sweeps_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, int own_lo,
                                         int own_hi, const double* rho, const double* v_in, double* v_out,
                                         double* scratch, int sweeps, double* diffs) {
    return guard(ctx, [&] {
        NEED(ctx && rho && v_in && v_out && scratch && (diffs || sweeps == 0), "NULL argument");
        NEED(v_in != v_out && v_in != scratch && v_out != scratch && rho != v_in && rho != v_out && rho != scratch,
             "rho, v_in, v_out and scratch must be distinct");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::zslab_jacobi_sweeps(ctx, G, z_lo, z_hi, own_lo, own_hi, rho, v_in, v_out, scratch, sweeps, diffs);
        dftb::sync(ctx);
    });
}

dft_status_t dft_zslab_hamiltonian_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, const double* V,
                                       const double* psi, double* hpsi, int nbands, long ld) {
    return guard(ctx, [&] {
        NEED(ctx && V && psi && hpsi, "NULL argument");
        NEED(nbands >= 0, "nbands must be >= 0");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::zslab_hamiltonian(ctx, G, z_lo, z_hi, V, psi, hpsi, nbands, ld);
    });
}

dft_status_t dft_zslab_xc_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, int own_lo, int own_hi,
                              dft_xc_kind kind, const double* na, const double* nb, double* va, double* vb,
                              double* exc_out) {
    return guard(ctx, [&] {
        NEED(ctx && na && nb, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        const double e = dftb::zslab_xc(ctx, G, z_lo, z_hi, own_lo, own_hi, (int)kind, na, nb, va, vb);
        dftb::sync(ctx);
        if (exc_out) *exc_out = e;
    });
}

dft_status_t dft_zslab_gram_dev(dft_context* ctx, const dft_grid* g, int z_lo, int z_hi, int own_lo, int own_hi,
                                const double* A, long lda, int ka, const double* B, long ldb, int kb, int precision,
                                double* C_host) {
    return guard(ctx, [&] {
        NEED(ctx && A && B && C_host, "NULL argument");
        NEED(ka > 0 && kb > 0, "bad sizes");
        const dftb::Grid G = dftb::make_grid(g);
        std::vector<double> C;
        dftb::zslab_gram(ctx, G, z_lo, z_hi, own_lo, own_hi, A, lda, ka, B, ldb, kb, precision, C);
        std::copy(C.begin(), C.end(), C_host);
    });
}

dft_status_t dft_hartree_monopole_dev(dft_context* ctx, const dft_grid* g, const double* rho, double* vh, double tol,
                                      long max_sweeps, long* sweeps_out, double* last_diff_out) {
    return guard(ctx, [&] {
        NEED(ctx && rho && vh, "NULL argument");
        NEED(rho != vh, "rho and vh must not alias");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::monopole_width(G);
        double *rp = nullptr, *vc = nullptr, *vp = nullptr;
        auto release = [&] {
            cudaFree(rp);
            cudaFree(vc);
            cudaFree(vp);
        };
        try {
            DFT_CUDA(cudaMalloc(&rp, sizeof(double) * (size_t)G.N));
            DFT_CUDA(cudaMalloc(&vc, sizeof(double) * (size_t)G.N));
            DFT_CUDA(cudaMalloc(&vp, sizeof(double) * (size_t)G.N));
            dftb::monopole_prepare(ctx, G, rho, rp, vc);
            dftb::JacobiResult r = dftb::hartree(ctx, G, rp, vp, tol, max_sweeps, nullptr, true);
            dftb::add_into(ctx, G.N, vp, vc, vh);
            dftb::sync(ctx);
            if (sweeps_out) *sweeps_out = r.sweeps;
            if (last_diff_out) *last_diff_out = r.last_diff;
        } catch (...) {
            release();
            throw;
        }
        release();
    });
}

dft_status_t dft_hartree_energy_dev(dft_context* ctx, const dft_grid* g, const double* rho, const double* vh,
                                    double* energy_out) {
    return guard(ctx, [&] {
        NEED(ctx && rho && vh && energy_out, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        *energy_out = 0.5 * dftb::dot(ctx, G.N, rho, vh) * G.dV;
    });
}

dft_status_t dft_xc_dev(dft_context* ctx, const dft_grid* g, dft_xc_kind kind, const double* na, const double* nb,
                        double* va, double* vb, double* exc_out) {
    return guard(ctx, [&] {
        NEED(ctx && na && nb, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        const double e = dftb::xc(ctx, G, (int)kind, na, nb, va, vb, exc_out != nullptr);
        dftb::sync(ctx);
        if (exc_out) *exc_out = e;
    });
}

dft_status_t dft_xc_evaluate_dev(dft_context* ctx, dft_xc_kind kind, long m, const double* na, const double* nb,
                                 const double* ga, const double* gb, double* out5) {
    return guard(ctx, [&] {
        NEED(ctx && na && nb && ga && gb && out5, "NULL argument");
        NEED(m >= 0, "m must be >= 0");
        dftb::xc_evaluate(ctx, (int)kind, m, na, nb, ga, gb, out5);
    });
}

dft_status_t dft_spin_density_dev(dft_context* ctx, long npoints, const double* psi, int nbands, long ld,
                                  const double* occ, double* out) {
    return guard(ctx, [&] {
        NEED(ctx && psi && occ && out, "NULL argument");
        NEED(nbands > 0, "La lista de orbitales moleculares no puede estar vacia.");
        NEED(npoints > 0 && ld >= npoints, "bad sizes");
        dftb::spin_density(ctx, npoints, psi, nbands, ld, occ, out);
    });
}

dft_status_t dft_kinetic_energy_dev(dft_context* ctx, const dft_grid* g, const double* psi, int nbands, long ld,
                                    const double* occ, double* energy_out) {
    return guard(ctx, [&] {
        NEED(ctx && psi && occ && energy_out, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        NEED(ld >= G.N, "ld must be >= nx*ny*nz");
        *energy_out = dftb::kinetic_energy(ctx, G, psi, nbands, ld, occ);
    });
}

dft_status_t dft_nuclear_potential_dev(dft_context* ctx, const dft_grid* g, int nnuc, const int* Z,
                                       const double* xyz, double* vext) {
    return guard(ctx, [&] {
        NEED(ctx && Z && xyz && vext, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::nuclear_potential(ctx, G, nnuc, Z, xyz, vext);
    });
}

dft_status_t dft_solve_orbitals_dev(dft_context* ctx, const dft_grid* g, const double* V, int nocc, int nbands,
                                    double* psi, long ld, int init, double* eig, const dft_eig_opts* opts,
                                    int* iterations_out) {
    return guard(ctx, [&] {
        NEED(ctx && V && psi && eig, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::EigOpts o;
        if (opts) {
            if (opts->tol > 0) o.tol = opts->tol;
            if (opts->max_iterations > 0) o.max_iterations = opts->max_iterations;
            if (opts->max_subspace >= 2) o.max_subspace = opts->max_subspace;
            o.precond_steps = opts->preconditioner;
            o.precond_net = opts->preconditioner_net;
            o.mixed_precision = opts->mixed_precision;
            o.verbose = opts->verbose;
        }
        const int it = dftb::solve_orbitals(ctx, G, V, nocc, nbands, psi, ld, init != 0, eig, nullptr, o);
        if (iterations_out) *iterations_out = it;
    });
}

dft_status_t dft_rotate_dev(dft_context* ctx, const dft_grid* g, const double* V, long ldv, int k, const double* Y,
                            int m, double* X, long ldx, int precision) {
    return guard(ctx, [&] {
        NEED(ctx && V && Y && X, "NULL argument");
        NEED(k >= 0 && m >= 0, "k and m must be >= 0");
        const dftb::Grid G = dftb::make_grid(g);
        NEED(ldv >= G.N && ldx >= G.N, "leading dimensions must be >= N");
        std::vector<double> Yv(Y, Y + (size_t)k * m);
        if (precision) dftb::rotate_tc(ctx, G, V, ldv, k, Yv, m, X, ldx);
        else dftb::rotate(ctx, G, V, ldv, k, Yv, m, X, ldx, 1.0, 0.0);
        dftb::sync(ctx);
    });
}

dft_status_t dft_screened_poisson_dev(dft_context* ctx, const dft_grid* g, const double* src, double* x, double q2,
                                      int cycles) {
    return guard(ctx, [&] {
        NEED(ctx && src && x, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::screened_poisson_vcycle(ctx, G, src, 1, q2, x, G.N, cycles);
        dftb::sync(ctx);
    });
}

dft_status_t dft_gram_dev(dft_context* ctx, const dft_grid* g, const double* A, long lda, int ka, const double* B,
                          long ldb, int kb, int precision, double* C_host) {
    return guard(ctx, [&] {
        NEED(ctx && A && B && C_host, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        NEED(ka > 0 && kb > 0 && lda >= G.N && ldb >= G.N, "bad sizes");
        std::vector<double> C;
        if (precision == 1) dftb::gram_tc(ctx, G, A, lda, ka, B, ldb, kb, C);
        else dftb::gram_fp64(ctx, G, A, lda, ka, B, ldb, kb, C);
        std::copy(C.begin(), C.end(), C_host);
    });
}

void dft_scf_default_options(dft_scf_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->max_iterations = 250;        // DFTConstants.h:13
    o->energy_tol = 1.0e-11;        // DFTConstants.h:16
    o->density_tol = 1.0e-9;        // DFTConstants.h:15
    o->ks_tol = 1.0e-7;             // DFTConstants.h:17
    o->stop_abs_de = 0.0;
    o->poisson_tol = 1.0e-8;        // HartreePotentialMolecule.cpp:15
    o->poisson_max_sweeps = 10000;  // HartreePotentialMolecule.cpp:14
    o->extra_bands = 3;
    o->eig.tol = 1.0e-7;            // EigenvalueSolverMolecule.cpp:19
    o->eig.max_iterations = 2000;
    o->eig.max_subspace = 3;
    o->eig.verbose = 0;
    o->eig.preconditioner = 4;
    o->verbose = 0;
}

dft_status_t dft_scf_molecule(dft_context* ctx, const dft_grid* g, int nnuc, const int* Z, const double* xyz,
                              int charge, int multiplicity, dft_xc_kind kind, const dft_scf_opts* opts,
                              dft_scf_result* result) {
    return guard(ctx, [&] {
        NEED(ctx && Z && xyz && result, "NULL argument");
        dftb::scf_molecule(ctx, g, nnuc, Z, xyz, charge, multiplicity, (int)kind, opts, result);
    });
}

dft_status_t dft_solve_atoms(dft_context* ctx, int nruns, const int* Z, const int* kinds, long points, double rmax,
                             dft_atom_result* results) {
    return guard(ctx, [&] {
        NEED(ctx && Z && kinds && results, "NULL argument");
        NEED(nruns > 0, "nruns must be > 0");
        dftb::solve_atoms(ctx, nruns, Z, kinds, points, rmax, results);
    });
}

}  // extern "C"

// ---------------------------------------------------------------- learned Poisson start --
dft_status_t dft_pnet_create(dft_context* ctx, int in_channels, unsigned long long seed, dft_pnet** out) {
    return guard(ctx, [&] {
        NEED(ctx && out, "NULL argument");
        *out = dftb::pnet_create(ctx, in_channels, seed);
    });
}

dft_status_t dft_pnet_destroy(dft_pnet* net) {
    return guard(nullptr, [&] { dftb::pnet_destroy(net); });
}

dft_status_t dft_pnet_num_params(const dft_pnet* net, size_t* n) {
    return guard(nullptr, [&] {
        NEED(net && n, "NULL argument");
        *n = dftb::pnet_num_params(net);
    });
}

dft_status_t dft_pnet_get_params(dft_context* ctx, dft_pnet* net, float* host, size_t n) {
    return guard(ctx, [&] {
        NEED(ctx && net && host, "NULL argument");
        NEED(n == dftb::pnet_num_params(net), "parameter count mismatch");
        dftb::pnet_get_params(ctx, net, host);
    });
}

dft_status_t dft_pnet_set_params(dft_context* ctx, dft_pnet* net, const float* host, size_t n) {
    return guard(ctx, [&] {
        NEED(ctx && net && host, "NULL argument");
        NEED(n == dftb::pnet_num_params(net), "parameter count mismatch");
        dftb::pnet_set_params(ctx, net, host);
    });
}

dft_status_t dft_pnet_loss_grad(dft_context* ctx, dft_pnet* net, int nx, int ny, int nz, const float* x,
                                const float* t, double* loss, float* grad, float* y) {
    return guard(ctx, [&] {
        NEED(ctx && net && x && t, "NULL argument");
        dftb::pnet_loss_grad(ctx, net, nx, ny, nz, x, t, loss, grad, y);
    });
}

dft_status_t dft_poisson_start_dev(dft_context* ctx, const dft_grid* g, dft_pnet* net, const double* rho,
                                   double* vstart, int multigrid_cycles, dft_poisson_start_info* info) {
    return guard(ctx, [&] {
        NEED(ctx && rho && vstart, "NULL argument");
        NEED(rho != vstart, "rho and vstart must not alias");
        NEED(multigrid_cycles >= 0, "multigrid_cycles must be >= 0");
        const dftb::Grid G = dftb::make_grid(g);
        dftb::PoissonGuessInfo pi;
        dftb::poisson_start(ctx, net, G, rho, vstart, multigrid_cycles, &pi);
        dftb::sync(ctx);
        if (info) {
            info->coarse_cycles = pi.coarse_cycles;
            info->multigrid_cycles = pi.cycles;
            info->residual = pi.residual;
            info->scale = pi.scale;
        }
    });
}

dft_status_t dft_synthetic_density_dev(dft_context* ctx, const dft_grid* g, unsigned long long seed, int kmin,
                                       int kmax, double wmin, double wmax, int ne_min, int ne_max, double* rho,
                                       int* ne_out) {
    return guard(ctx, [&] {
        NEED(ctx && rho, "NULL argument");
        const dftb::Grid G = dftb::make_grid(g);
        const int ne = dftb::synthetic_density(ctx, G, seed, kmin, kmax, wmin, wmax, ne_min, ne_max, rho);
        dftb::sync(ctx);
        if (ne_out) *ne_out = ne;
    });
}

dft_status_t dft_pnet_train_poisson(dft_context* ctx, dft_pnet* net, const dft_pnet_train_opts* opts,
                                    dft_pnet_train_report* report) {
    return guard(ctx, [&] {
        NEED(ctx && net && opts && report, "NULL argument");
        dftb::pnet_train_poisson(ctx, net, opts, report);
    });
}

dft_status_t dft_pnet_train_preconditioner(dft_context* ctx, dft_pnet* net, const dft_grid* g, const double* V,
                                           int nocc, int nbands, const dft_pnet_train_opts* opts,
                                           dft_pnet_train_report* report) {
    return guard(ctx, [&] {
        NEED(ctx && net && g && V && opts && report, "NULL argument");
        NEED(nocc > 0 && nbands >= nocc, "need 0 < nocc <= nbands");
        dftb::pnet_train_precond(ctx, net, dftb::make_grid(g), V, nocc, nbands, opts, report);
    });
}
