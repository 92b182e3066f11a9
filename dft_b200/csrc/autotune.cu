// Launch-shape autotuner.  Several kernels here come in variants that give bit-identical
// results and differ only in speed, which depends on the grid and the band count: the H psi
// kernel marches 1, 2 or 4 bands per thread, and the Jacobi Poisson solve runs one sweep per
// launch, 2/4/8 temporally blocked sweeps per launch, the whole solve in one persistent
// cooperative launch, or the whole solve in the shared memory of a 16-block cluster.  The
// autotuner times every variant on the caller's grid (CUDA events on the context's stream,
// after one warm-up call each) and remembers the fastest per grid in the context; kernels on
// that grid use it wherever the corresponding tuning knob is 0 (auto).  A repeated call for a
// grid already tuned costs nothing.
#include <algorithm>
#include <vector>

#include "ops.h"

namespace dftb {

namespace {

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    Events() {
        DFT_CUDA(cudaEventCreate(&a));
        DFT_CUDA(cudaEventCreate(&b));
    }
    ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

// milliseconds of fn() on the context's stream: one warm-up call, then the fastest of reps
template <typename F>
double time_ms(dft_context* ctx, Events& ev, int reps, F&& fn) {
    fn();
    sync(ctx);
    double best = 1e300;
    for (int r = 0; r < reps; ++r) {
        DFT_CUDA(cudaEventRecord(ev.a, ctx->stream));
        fn();
        DFT_CUDA(cudaEventRecord(ev.b, ctx->stream));
        DFT_CUDA(cudaEventSynchronize(ev.b));
        float ms = 0.f;
        DFT_CUDA(cudaEventElapsedTime(&ms, ev.a, ev.b));
        best = std::min(best, (double)ms);
    }
    return best;
}

}  // namespace

void autotune(dft_context* ctx, const Grid& g, int nbands, dft_autotune_report* rep) {
    if (nbands < 1) fail(DFT_INVALID_ARGUMENT, "nbands must be >= 1");
    dft_autotune_report r{};
    const std::array<long long, 3> key{g.nx, g.ny, g.nz};
    auto hit = ctx->tuned.find(key);
    if (hit != ctx->tuned.end()) {
        r.hpsi_bands_per_thread = hit->second[0];
        r.jacobi_sweeps_per_launch = hit->second[1];
        r.hpsi_variant = hit->second[2];
        r.hpsi_zchunk = hit->second[3];
        r.cached = 1;
        if (rep) *rep = r;
        return;
    }
    // the knobs are set per variant while timing and put back afterwards
    const int keep_bpt = ctx->hpsi_bands_per_thread, keep_spl = ctx->jacobi_sweeps_per_launch;
    const int keep_var = ctx->hpsi_variant;
    struct Restore {
        dft_context* c;
        int b, s, v;
        ~Restore() {
            c->hpsi_bands_per_thread = b;
            c->jacobi_sweeps_per_launch = s;
            c->hpsi_variant = v;
        }
    } restore{ctx, keep_bpt, keep_spl, keep_var};
    Events ev;
    const long long N = g.N;
    // timing buffers: at most 16 bands (the per-band cost is what differs), zero fields (the
    // arithmetic of these kernels does not depend on the values)
    const int tb = std::min(nbands, 16);
    double* buf = nullptr;
    DFT_CUDA(cudaMalloc(&buf, sizeof(double) * (size_t)N * (2 * tb + 3)));
    struct Free {
        double* p;
        ~Free() {
            if (p) cudaFree(p);
        }
    } free_buf{buf};
    DFT_CUDA(cudaMemsetAsync(buf, 0, sizeof(double) * (size_t)N * (2 * tb + 3), ctx->stream));
    double *V = buf, *psi = buf + N, *hpsi = psi + (size_t)tb * N, *rho = hpsi + (size_t)tb * N, *vh = rho + N;
    // ---- H psi: bands per thread
    const int bpt[3] = {1, 2, 4};
    int best_bpt = 1, best_var = 0;
    double best = 1e300;
    ctx->hpsi_variant = 0;
    for (int i = 0; i < 3; ++i) {
        if (bpt[i] > tb && i > 0) {
            r.hpsi_ms[i] = -1.0;
            continue;
        }
        ctx->hpsi_bands_per_thread = bpt[i];
        r.hpsi_ms[i] = time_ms(ctx, ev, 3, [&] { apply_hamiltonian(ctx, g, V, psi, hpsi, tb, N); });
        if (r.hpsi_ms[i] < best) best = r.hpsi_ms[i], best_bpt = bpt[i];
    }
    // the TMA plane ring, bands per block (where the grid and the block allow it)
    const int nbc[4] = {1, 2, 4, 8};
    const bool tma_ok = hpsi_tma_eligible(g, psi, N);
    ctx->hpsi_variant = 2;
    for (int i = 0; i < 4; ++i) {
        if (!tma_ok || (nbc[i] > tb && i > 0)) {
            r.hpsi_tma_ms[i] = -1.0;
            continue;
        }
        ctx->hpsi_bands_per_thread = nbc[i];
        r.hpsi_tma_ms[i] = time_ms(ctx, ev, 3, [&] { apply_hamiltonian(ctx, g, V, psi, hpsi, tb, N); });
        if (r.hpsi_tma_ms[i] < best) best = r.hpsi_tma_ms[i], best_bpt = nbc[i], best_var = 2;
    }
    check_device_status(ctx, "autotune");
    // the prefetching single-band march
    ctx->hpsi_variant = 3;
    ctx->hpsi_bands_per_thread = 1;
    r.hpsi_prefetch_ms = time_ms(ctx, ev, 3, [&] { apply_hamiltonian(ctx, g, V, psi, hpsi, tb, N); });
    if (r.hpsi_prefetch_ms < best) best = r.hpsi_prefetch_ms, best_bpt = 1, best_var = 3;
    // the march length per block of the chosen register march (the auto choice is zc = 0)
    int best_zc = 0;
    if (best_var == 0 || best_var == 3) {
        const int keep_zc = ctx->hpsi_zchunk;
        ctx->hpsi_variant = best_var;
        ctx->hpsi_bands_per_thread = best_bpt;
        const int zcs[5] = {16, 32, 64, 96, 192};
        for (int i = 0; i < 5; ++i) {
            if (zcs[i] > g.nz) {
                r.hpsi_zchunk_ms[i] = -1.0;
                continue;
            }
            ctx->hpsi_zchunk = zcs[i];
            r.hpsi_zchunk_ms[i] = time_ms(ctx, ev, 3, [&] { apply_hamiltonian(ctx, g, V, psi, hpsi, tb, N); });
            if (r.hpsi_zchunk_ms[i] < best) best = r.hpsi_zchunk_ms[i], best_zc = zcs[i];
        }
        ctx->hpsi_zchunk = keep_zc;
    } else {
        for (double& v : r.hpsi_zchunk_ms) v = -1.0;
    }
    r.hpsi_zchunk = best_zc;
    ctx->hpsi_variant = 0;
    r.hpsi_bands_per_thread = best_bpt;
    r.hpsi_variant = best_var;
    // ---- Jacobi: sweeps per launch; tol = 0 never stops, so each call runs exactly `sweeps`
    const int spl[6] = {-2, -1, 1, 2, 4, 8};
    const long sweeps = 64;
    int best_spl = 1;
    best = 1e300;
    for (int i = 0; i < 6; ++i) {
        ctx->jacobi_sweeps_per_launch = spl[i];
        double ms = -1.0;
        try {
            ms = time_ms(ctx, ev, 2, [&] { hartree(ctx, g, rho, vh, 0.0, sweeps); });
        } catch (const Error& e) {
            if (e.status != DFT_INVALID_ARGUMENT) throw;  // the cluster variant does not fit this grid
        }
        r.jacobi_us_per_sweep[i] = ms < 0 ? -1.0 : 1e3 * ms / sweeps;
        if (ms >= 0 && ms < best) best = ms, best_spl = spl[i];
    }
    r.jacobi_sweeps_per_launch = best_spl;
    sync(ctx);
    ctx->tuned[key] = {best_bpt, best_spl, best_var, best_zc};
    if (rep) *rep = r;
}

}  // namespace dftb
