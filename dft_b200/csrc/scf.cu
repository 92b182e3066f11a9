// Molecular SCF driver: the reference loop (SelfConsistentFieldMolecule.cpp:50-561 with
// executeMolecularSCFIteration, MolecularSCFIteration.cpp:12-252) over device-resident
// fields.  Densities, potentials and orbitals never leave HBM; only scalars (energies,
// norms, the small projected matrices) come back to the host.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <limits>
#include <string>
#include <vector>

#include "neural.h"
#include "ops.h"

namespace dftb {

namespace {

using Clock = std::chrono::steady_clock;
inline double ms_since(Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

// An SCF's device buffer, taken from and given back to the context's pool of released
// buffers (exact sizes); everything stays stream-ordered on the context's one stream, so a
// buffer handed to the next SCF is used only after this SCF's kernels.  The pool keeps at most
// 32 GiB; beyond that a released buffer is freed.
struct DevBuf {
    dft_context* c = nullptr;
    double* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(dft_context* ctx, size_t n) : c(ctx), bytes(n * sizeof(double)) {
        if (!n) return;
        auto it = c->buf_pool.find(bytes);
        if (it != c->buf_pool.end()) {
            p = (double*)it->second;
            c->buf_pool.erase(it);
            c->buf_pool_bytes -= bytes;
        } else {
            DFT_CUDA(cudaMalloc(&p, bytes));
        }
    }
    void release() {
        if (!p) return;
        if (c && c->buf_pool_bytes + bytes <= (32ULL << 30)) {
            c->buf_pool.emplace(bytes, p);
            c->buf_pool_bytes += bytes;
        } else {
            cudaFree(p);
        }
        p = nullptr;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

// per-block sums of psi^2 over points within w bohr of a face, and over all points
__global__ void wall_weight_kernel(Grid g, const double* __restrict__ psi, double w, double* __restrict__ partial) {
    __shared__ double sh[2][8];
    double a = 0.0, t = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const double x = g.xmin + i * g.dx, y = g.ymin + j * g.dy, z = g.zmin + k * g.dz;
        const double d = fmin(fmin(fmin(x - g.xmin, g.xmax - x), fmin(y - g.ymin, g.ymax - y)),
                              fmin(z - g.zmin, g.zmax - z));
        const double v = psi[p] * psi[p];
        t += v;
        if (d < w) a += v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = a;
        sh[1][threadIdx.x >> 5] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, st = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) sa += sh[0][q], st += sh[1][q];
        partial[2 * blockIdx.x] = sa;
        partial[2 * blockIdx.x + 1] = st;
    }
}

// fraction of |psi|^2 within w bohr of a face (diagnostics)
double wall_fraction(dft_context* ctx, const Grid& g, const double* psi, double w) {
    const int nb = std::max(1, std::min((int)((g.N + 255) / 256), ctx->num_sms * 4));
    double* partial = (double*)ws_get(ctx, WS_SCF3, sizeof(double) * 2 * (size_t)nb);
    wall_weight_kernel<<<nb, 256, 0, ctx->stream>>>(g, psi, w, partial);
    DFT_LAUNCH_CHECK();
    std::vector<double> h(2 * (size_t)nb);
    DFT_CUDA(cudaMemcpyAsync(h.data(), partial, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    double a = 0.0, t = 0.0;
    for (int q = 0; q < nb; ++q) a += h[2 * q], t += h[2 * q + 1];
    return t > 0.0 ? a / t : 0.0;
}

}  // namespace

void scf_molecule(dft_context* ctx, const dft_grid* grid, int nnuc, const int* Z, const double* xyz, int charge,
                  int multiplicity, int kind, const dft_scf_opts* opts, dft_scf_result* res) {
    const auto t_start = Clock::now();
    const Grid g = make_grid(grid);
    if (!res) fail(DFT_INVALID_ARGUMENT, "result is NULL");
    if (kind != DFT_XC_PZ81 && kind != DFT_XC_PBE96) fail(DFT_INVALID_ARGUMENT, "unknown functional kind %d", kind);
    dft_scf_opts o;
    if (opts) o = *opts;
    else dft_scf_default_options(&o);
    // ---- input checks, reference SelfConsistentFieldMolecule.cpp:58-127 -----------------
    if (nnuc <= 0) fail(DFT_INVALID_ARGUMENT, "La molecula debe contener al menos un nucleo.");
    if (multiplicity < 1) fail(DFT_INVALID_ARGUMENT, "La multiplicidad electronica debe ser al menos 1.");
    int nuclear = 0;
    for (int a = 0; a < nnuc; ++a) {
        if (Z[a] <= 0) fail(DFT_INVALID_ARGUMENT, "Atomic number must be greater than zero.");
        nuclear += Z[a];
    }
    const int ne = nuclear - charge;
    if (ne < 0) fail(DFT_INVALID_ARGUMENT, "La carga molecular produce un numero negativo de electrones.");
    if (ne == 0) fail(DFT_INVALID_ARGUMENT, "El SCF molecular requiere al menos un electron.");
    const int sd = multiplicity - 1;
    if (sd > ne) fail(DFT_INVALID_ARGUMENT, "La multiplicidad electronica es incompatible con el numero de electrones.");
    if ((ne - sd) % 2 != 0)
        fail(DFT_INVALID_ARGUMENT, "La multiplicidad electronica es incompatible con la paridad del numero de electrones.");
    const int na = (ne + sd) / 2, nb = (ne - sd) / 2;
    const bool closed = multiplicity == 1;
    // zero beta electrons: the reference's solveMolecularOrbitals(0 orbitals) throws (:1240-1246)
    if (nb == 0) fail(DFT_INVALID_ARGUMENT, "El numero de orbitales debe ser mayor que cero.");

    const long long N = g.N, ld = N;
    const int extra = std::max(0, o.extra_bands);
    const int bands_a = (int)std::min<long long>(na + extra, N);
    const int bands_b = (int)std::min<long long>(nb + extra, N);
    EigOpts eo;
    eo.tol = o.eig.tol > 0 ? o.eig.tol : 1e-7;
    eo.max_iterations = o.eig.max_iterations > 0 ? o.eig.max_iterations : 2000;
    eo.max_subspace = o.eig.max_subspace >= 2 ? o.eig.max_subspace : 3;
    eo.precond_steps = o.eig.preconditioner;
    eo.precond_net = o.eig.preconditioner_net;
    eo.mixed_precision = o.eig.mixed_precision;
    eo.verbose = o.eig.verbose;

    const int pstart = o.poisson_start;
    if (pstart < DFT_POISSON_COLD || pstart > DFT_POISSON_MULTIGRID)
        fail(DFT_INVALID_ARGUMENT, "unknown poisson_start %d", pstart);
    if (pstart == DFT_POISSON_NETWORK && !o.poisson_net)
        fail(DFT_INVALID_ARGUMENT, "poisson_start DFT_POISSON_NETWORK needs poisson_net");

    DevBuf vext(ctx, N), da(ctx, N), db(ctx, N), rho(ctx, N), vh(ctx, N), vxa(ctx, N), vxb(ctx, N), va(ctx, N),
        vb(ctx, N), oa(ctx, N), ob(ctx, N), orho(ctx, N), ovh(ctx, N);
    DevBuf vstart(ctx, pstart >= DFT_POISSON_NETWORK ? (size_t)N : 0);
    dft_pnet* net = pstart == DFT_POISSON_COARSE ? nullptr : o.poisson_net;
    // Poisson solve of density d into v with the chosen start; `have_prev` says whether v
    // still holds this slot's potential from the previous iteration.
    // Monopole faces: the zero-face solve runs on (rho', V') per slot, V_H = V' + V_c.
    const bool monopole = o.hartree_boundary == 1;
    if (monopole) monopole_width(g);  // the origin must lie well inside the box
    DevBuf mrho(ctx, monopole ? (size_t)N : 0), mvc(ctx, monopole ? (size_t)N : 0), mvp0(ctx, monopole ? (size_t)N : 0),
        mvp1(ctx, monopole ? (size_t)N : 0);
    int last_cycles = 0;  // multigrid cycles of the last solve
    // Jacobi spectral radius of the grid: a max|dV| stop at tol leaves ~tol / (1 - rho) of error
    const double rho_j = (g.ix2 * std::cos(3.14159265358979323846 / (g.nx - 1)) +
                          g.iy2 * std::cos(3.14159265358979323846 / (g.ny - 1)) +
                          g.iz2 * std::cos(3.14159265358979323846 / (g.nz - 1))) /
                         (g.ix2 + g.iy2 + g.iz2);
    const double fixed_scale = std::max(1.0 - rho_j, 1e-6);
    if (o.poisson_fixed_point != 0 && o.poisson_fixed_point != 1)
        fail(DFT_INVALID_ARGUMENT, "unknown poisson_fixed_point %d", o.poisson_fixed_point);
    auto poisson = [&](const double* d_in, double* v_out, bool have_prev, double tol = -1.0) {
        // multigrid target: half the Jacobi stop, scaled by 1 - rho with poisson_fixed_point
        const double ptol = tol > 0.0 ? tol : o.poisson_tol * (o.poisson_fixed_point ? fixed_scale : 1.0);
        last_cycles = 0;
        const double* d = d_in;
        double* v = v_out;
        if (monopole) {
            monopole_prepare(ctx, g, d_in, mrho.p, mvc.p);
            d = mrho.p;
            v = v_out == vh.p ? mvp0.p : mvp1.p;
        }
        const double* start = nullptr;
        if (pstart == DFT_POISSON_MULTIGRID) {
            const auto t0 = Clock::now();
            int cyc = 0;
            double res = 0.0;
            if (have_prev) {
                DFT_CUDA(cudaMemcpyAsync(vstart.p, v, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
                // the multigrid keeps the start's faces; the zero-face part of the monopole
                // boundary must start from exactly zero faces (a start combined from potentials
                // of slightly different total charge carries face values of order dQ/|r|)
                if (monopole) zero_faces(ctx, g, vstart.p);
                cyc = multigrid(ctx, g, d, vstart.p, 0.5 * ptol, 40, &res);
            } else {
                PoissonGuessInfo info;
                poisson_start(ctx, net, g, d, vstart.p, 40, &info);
                cyc = info.cycles;
                res = info.residual;
            }
            last_cycles = cyc;
            if (o.verbose > 1)
                fprintf(stderr, "[poisson] multigrid %d cycles, next Jacobi update %.3e, %.2f ms\n", cyc, res,
                        ms_since(t0));
            start = vstart.p;
        } else if ((pstart == DFT_POISSON_PREVIOUS || pstart == DFT_POISSON_HYBRID) && have_prev) {
            start = v;
        } else if (pstart >= DFT_POISSON_NETWORK) {
            poisson_start(ctx, net, g, d, vstart.p, 0, nullptr);
            start = vstart.p;
        }
        // the Jacobi stop: the given tolerance, else the caller's (its rule is unchanged)
        const JacobiResult r = hartree(ctx, g, d, v, tol > 0.0 ? tol : o.poisson_tol, o.poisson_max_sweeps, start,
                                       monopole);
        if (monopole) add_into(ctx, N, v, mvc.p, v_out);
        return r;
    };
    DevBuf psia(ctx, (size_t)bands_a * ld), psib(ctx, closed ? 0 : (size_t)bands_b * ld);
    std::vector<double> eiga(bands_a), eigb(bands_b), resa(bands_a), resb(bands_b);
    std::vector<double> occa(bands_a, 0.0), occb(bands_b, 0.0);
    for (int i = 0; i < na; ++i) occa[i] = 1.0;  // buildSpinOccupations: one electron per orbital
    for (int i = 0; i < nb; ++i) occb[i] = 1.0;

    if (o.autotune) autotune(ctx, g, std::max(bands_a, bands_b), nullptr);
    nuclear_potential(ctx, g, nnuc, Z, xyz, vext.p);
    // NuclearRepulsion::calculate (NuclearRepulsion.cpp:6-54)
    double enn = 0.0;
    for (int a = 0; a < nnuc; ++a)
        for (int c = a + 1; c < nnuc; ++c) {
            const double dx = xyz[3 * a] - xyz[3 * c], dy = xyz[3 * a + 1] - xyz[3 * c + 1],
                         dz = xyz[3 * a + 2] - xyz[3 * c + 2];
            const double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 == 0.0) fail(DFT_SINGULAR, "NuclearRepulsion is undefined for coincident nuclei.");
            enn += (double)Z[a] * (double)Z[c] / std::sqrt(d2);
        }

    // ---- initial densities ------------------------------------------------------------
    if (o.initial_density != 0 && o.initial_density != 1)
        fail(DFT_INVALID_ARGUMENT, "unknown initial_density %d", o.initial_density);
    // superposed radial atoms (option): densities now, atomic orbitals as the first eigensolve's
    // start basis (both spins), freed after the first iteration
    const bool atoms_start = o.initial_density == 1;
    if (o.hartree_boundary != 0 && o.hartree_boundary != 1)
        fail(DFT_INVALID_ARGUMENT, "unknown hartree_boundary %d", o.hartree_boundary);
    int nao = 0;
    DevBuf aobuf;
    if (atoms_start) {
        const long long kcap = std::max<long long>(eo.max_subspace * (long long)std::max(bands_a, bands_b),
                                                   std::max(bands_a, bands_b) + 16LL) - 1;
        const int want = (int)std::min<long long>(atomic_orbital_count(nnuc, Z), kcap);
        if (want > 0) {
            DevBuf tmp(ctx, (size_t)want * ld);
            std::swap(aobuf.p, tmp.p);
            std::swap(aobuf.c, tmp.c);
            std::swap(aobuf.bytes, tmp.bytes);
        }
        nao = atomic_start(ctx, g, nnuc, Z, xyz, kind, na, nb, da.p, db.p, aobuf.p, ld, want);
    } else {
        // orbitals in the bare V_ext (MolecularSCFHelpers.cpp:515-579)
        solve_orbitals(ctx, g, vext.p, na, bands_a, psia.p, ld, false, eiga.data(), resa.data(), eo);
        spin_density(ctx, N, psia.p, bands_a, ld, occa.data(), da.p);
        if (closed) {
            DFT_CUDA(cudaMemcpyAsync(db.p, da.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
        } else {
            solve_orbitals(ctx, g, vext.p, nb, bands_b, psib.p, ld, false, eigb.data(), resb.data(), eo);
            spin_density(ctx, N, psib.p, bands_b, ld, occb.data(), db.p);
        }
    }

    // ---- Fermi-Dirac occupations (option; the reference fills the lowest levels) --------
    const double kt = o.smearing_kt;
    if (kt < 0.0 || !std::isfinite(kt)) fail(DFT_INVALID_ARGUMENT, "smearing_kt must be >= 0");
    // f_i = 1 / (1 + exp((e_i - mu) / kt)) with sum f_i = nel, mu by bisection; returns the
    // number of bands to converge tightly (every band with f_i > 1e-8, at least nel)
    auto fermi = [&](const std::vector<double>& e, int nel, std::vector<double>& f) {
        const int m = (int)e.size();
        if (nel >= m) {
            std::fill(f.begin(), f.end(), 1.0);
            return m;
        }
        double lo = *std::min_element(e.begin(), e.end()) - 40.0 * kt;
        double hi = *std::max_element(e.begin(), e.end()) + 40.0 * kt;
        auto count = [&](double mu) {
            double c = 0.0;
            for (int i = 0; i < m; ++i) {
                const double x = (e[i] - mu) / kt;
                c += x > 700.0 ? 0.0 : 1.0 / (1.0 + std::exp(x));
            }
            return c;
        };
        for (int k = 0; k < 200; ++k) {
            const double mid = 0.5 * (lo + hi);
            (count(mid) < nel ? lo : hi) = mid;
        }
        const double mu = 0.5 * (lo + hi);
        int nconv = nel;
        for (int i = 0; i < m; ++i) {
            const double x = (e[i] - mu) / kt;
            f[i] = x > 700.0 ? 0.0 : 1.0 / (1.0 + std::exp(x));
            if (f[i] > 1e-8) nconv = std::max(nconv, i + 1);
        }
        return nconv;
    };
    int nconv_a = na, nconv_b = nb;

    // ---- Pulay mixer state (option; the reference mixes linearly) -----------------------
    const int ns = closed ? 1 : 2;
    // defaults from a sweep over H2 48^3, H2O 128^3 and (H2O)_2 192^3: step 0.5 and 16 entries
    // took 11 / 21 / 41 iterations where 0.2 and 8 took 18 / 26 / more than 100
    const int pdepth = o.pulay_depth > 0 ? std::min(o.pulay_depth, 16) : 16;
    const double pbeta = o.pulay_beta > 0.0 ? o.pulay_beta : 0.5;
    if (o.mixer != 0 && o.mixer != 1) fail(DFT_INVALID_ARGUMENT, "unknown mixer %d", o.mixer);
    DevBuf phist(ctx, o.mixer == 1 ? (size_t)2 * pdepth * ns * N : 0);
    // Hartree start from the mixer (option): V_H is linear in the density, so the mixer's
    // combination of the stored V_H(n_in,i) and V_H(n_out,i) - V_H(n_in,i) is a start for the
    // next V_H(n_in) that is as close as those solves were (the unchanged stop rule ends it)
    if (o.poisson_predict < 0 || o.poisson_predict > 2)
        fail(DFT_INVALID_ARGUMENT, "unknown poisson_predict %d", o.poisson_predict);
    const bool vpredict = o.poisson_predict >= 1 && pstart != DFT_POISSON_COLD;
    // 2: also V_H(n_out) from V_H(n_in) + the previous iteration's V_H(n_out) - V_H(n_in)
    const bool vpredict_out = o.poisson_predict == 2 && pstart != DFT_POISSON_COLD;
    DevBuf vres(ctx, vpredict_out ? (size_t)N : 0);
    DevBuf vhist(ctx, vpredict && o.mixer == 1 ? (size_t)2 * pdepth * N : 0);
    DevBuf vtmp(ctx, vpredict && o.mixer == 1 && pdepth > 8 ? (size_t)N : 0);
    // Kerker screening of the total-charge residual (option; 0 = off, the reference's mixer)
    const double kq0 = o.kerker_q0;
    if (kq0 < 0.0 || !std::isfinite(kq0)) fail(DFT_INVALID_ARGUMENT, "kerker_q0 must be >= 0");
    const double kq2 = kq0 * kq0;
    DevBuf kbuf(ctx, kq0 > 0.0 ? (size_t)(ns + 2) * N : 0);
    std::vector<double> Bp((size_t)pdepth * pdepth, 0.0);
    int pcount = 0, phead = 0;
    auto pulay_mix = [&]() {
        const int slot = phead;
        double* hin = phist.p + (size_t)slot * 2 * ns * N;
        double* hres = hin + (size_t)ns * N;
        DFT_CUDA(cudaMemcpyAsync(hin, da.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
        sub(ctx, N, oa.p, da.p, hres);
        if (!closed) {
            DFT_CUDA(cudaMemcpyAsync(hin + N, db.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
            sub(ctx, N, ob.p, db.p, hres + N);
        }
        if (vpredict) {
            double* vin = vhist.p + (size_t)slot * 2 * N;
            DFT_CUDA(cudaMemcpyAsync(vin, vh.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
            sub(ctx, N, ovh.p, vh.p, vin + N);
        }
        phead = (phead + 1) % pdepth;
        pcount = std::min(pcount + 1, pdepth);
        for (int j = 0; j < pcount; ++j) {
            const double* rj = phist.p + (size_t)j * 2 * ns * N + (size_t)ns * N;
            const double v = dot(ctx, (long long)ns * N, hres, rj);
            Bp[(size_t)slot * pdepth + j] = Bp[(size_t)j * pdepth + slot] = v;
        }
        // minimise |sum c_i r_i| with sum c_i = 1: [B 1; 1 0][c; l] = [0; 1], Gaussian
        // elimination with partial pivoting; a singular system falls back to the newest entry
        const int m = pcount, M = m + 1;
        std::vector<double> A((size_t)M * M, 0.0), rhs(M, 0.0);
        double tr = 0.0;
        for (int i = 0; i < m; ++i) tr += Bp[(size_t)i * pdepth + i];
        for (int i = 0; i < m; ++i) {
            for (int j = 0; j < m; ++j) A[(size_t)i * M + j] = Bp[(size_t)i * pdepth + j];
            A[(size_t)i * M + i] += 1e-12 * tr;
            A[(size_t)i * M + m] = A[(size_t)m * M + i] = 1.0;
        }
        rhs[m] = 1.0;
        bool ok = true;
        for (int c = 0; c < M && ok; ++c) {
            int piv = c;
            for (int r = c + 1; r < M; ++r)
                if (std::fabs(A[(size_t)r * M + c]) > std::fabs(A[(size_t)piv * M + c])) piv = r;
            if (!(std::fabs(A[(size_t)piv * M + c]) > 1e-300)) {
                ok = false;
                break;
            }
            if (piv != c) {
                for (int k = 0; k < M; ++k) std::swap(A[(size_t)c * M + k], A[(size_t)piv * M + k]);
                std::swap(rhs[c], rhs[piv]);
            }
            for (int r = c + 1; r < M; ++r) {
                const double f = A[(size_t)r * M + c] / A[(size_t)c * M + c];
                for (int k = c; k < M; ++k) A[(size_t)r * M + k] -= f * A[(size_t)c * M + k];
                rhs[r] -= f * rhs[c];
            }
        }
        std::vector<double> cf(M, 0.0);
        if (ok) {
            for (int r = M - 1; r >= 0; --r) {
                double v = rhs[r];
                for (int k = r + 1; k < M; ++k) v -= A[(size_t)r * M + k] * cf[k];
                cf[r] = v / A[(size_t)r * M + r];
            }
            for (int i = 0; i < m; ++i) ok = ok && std::isfinite(cf[i]);
        }
        if (!ok) {
            std::fill(cf.begin(), cf.end(), 0.0);
            cf[slot] = 1.0;
        }
        double* dst[2] = {da.p, db.p};
        for (int sp = 0; sp < ns; ++sp) {
            const double* a[16];
            const double* r[16];
            for (int i = 0; i < m; ++i) {
                a[i] = phist.p + (size_t)i * 2 * ns * N + (size_t)sp * N;
                r[i] = a[i] + (size_t)ns * N;
            }
            if (kq0 > 0.0) {
                // n_in = sum c_i n_in,i + beta K(sum c_i r_i): the optimal residual screened
                combine(ctx, N, m, a, cf.data(), dst[sp]);
                combine(ctx, N, m, r, cf.data(), kbuf.p + (size_t)sp * N);
            } else {
                pulay_combine(ctx, N, m, a, r, cf.data(), pbeta, dst[sp]);
            }
        }
        if (kq0 > 0.0) {
            const double* rr[2] = {kbuf.p, kbuf.p + N};
            kerker_update(ctx, g, ns, dst, rr, kbuf.p + (size_t)ns * N, kbuf.p + (size_t)(ns + 1) * N, kq2, pbeta);
        }
        if (closed) DFT_CUDA(cudaMemcpyAsync(db.p, da.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
        if (vpredict) {
            // V = sum c_i (V_in,i + beta (V_out,i - V_in,i)); with Kerker screening the step's
            // screened part is not known and the unscreened one stands in (only a start)
            const double* a[16];
            double cv[16];
            for (int i = 0; i < m; ++i) a[i] = vhist.p + (size_t)i * 2 * N;
            if (2 * m <= 16) {
                for (int i = 0; i < m; ++i) {
                    a[m + i] = a[i] + N;
                    cv[i] = cf[i];
                    cv[m + i] = pbeta * cf[i];
                }
                combine(ctx, N, 2 * m, a, cv, vh.p);
            } else {
                combine(ctx, N, m, a, cf.data(), vh.p);
                for (int i = 0; i < m; ++i) {
                    a[i] += N;
                    cv[i] = pbeta * cf[i];
                }
                combine(ctx, N, m, a, cv, vtmp.p);
                add_into(ctx, N, vh.p, vtmp.p, vh.p);
            }
        }
    };

    // ---- SCF loop, constants SelfConsistentFieldMolecule.cpp:27-31 ----------------------
    double prevE = std::numeric_limits<double>::infinity();
    double prevD = std::numeric_limits<double>::infinity();
    double mixing = 0.25;  // DFTConstants::MIXING
    double E[6] = {0, 0, 0, 0, 0, 0};
    double effd = 0.0, resid = 0.0, dE = std::numeric_limits<double>::infinity();
    bool converged = false;
    int it = 0;
    std::vector<double> prev_eig;
    double deig = std::numeric_limits<double>::infinity();
    res->history_len = 0;
    // convergence analysis (MolecularSCFConvergenceAnalysis, reference MolecularSCFHelpers.h:47-72)
    res->last_energy_criterion_iteration = res->last_density_criterion_iteration = res->last_ks_criterion_iteration = 0;
    res->min_energy_difference = res->min_density_difference = res->min_ks_residual =
        std::numeric_limits<double>::infinity();
    res->final_mixing = 0.0;
    // JSON-lines log (option): one object per iteration and a final result line
    FILE* log = nullptr;
    if (o.log_path) {
        log = std::fopen(o.log_path, "w");
        if (!log) fail(DFT_INVALID_ARGUMENT, "cannot open the SCF log file '%s'", o.log_path);
    }
    struct LogCloser {
        FILE*& f;
        ~LogCloser() {
            if (f) std::fclose(f);
        }
    } log_closer{log};
    auto jnum = [](double v) {  // JSON has no inf/nan
        char b[40];
        if (std::isfinite(v)) std::snprintf(b, sizeof b, "%.17g", v);
        else std::snprintf(b, sizeof b, "null");
        return std::string(b);
    };
    auto jlevels = [&](const std::vector<double>& e, int nocc) {
        std::string r = "[";
        for (int i = std::max(0, nocc - 3); i < std::min((int)e.size(), nocc + 3); ++i)
            r += (r.size() > 1 ? "," : "") + jnum(e[i]);
        return r + "]";
    };
    std::vector<double> Ta(bands_a), Tb(bands_b);
    for (it = 1; it <= o.max_iterations; ++it) {
        const auto t_it = Clock::now();
        dft_scf_iteration rec{};
        rec.iteration = it;
        const double imix = mixing;
        // n -> V_H(n) (MolecularSCFIteration.cpp:45-66)
        auto t0 = Clock::now();
        add2(ctx, N, da.p, db.p, rho.p);
        JacobiResult jin = poisson(rho.p, vh.p, it > 1);
        sync(ctx);
        rec.ms_hartree = ms_since(t0);
        rec.poisson_sweeps_in = jin.sweeps;
        rec.poisson_cycles_in = last_cycles;
        // v_xc (:68-90): the closed-shell shortcut reuses alpha
        t0 = Clock::now();
        xc(ctx, g, kind, da.p, db.p, vxa.p, closed ? nullptr : vxb.p, false);
        add3(ctx, N, vext.p, vh.p, vxa.p, va.p);
        if (!closed) add3(ctx, N, vext.p, vh.p, vxb.p, vb.p);
        sync(ctx);
        rec.ms_xc = ms_since(t0);
        // orbitals (:117-144), warm-started from the previous iteration
        t0 = Clock::now();
        EigOpts ek = eo;
        if (o.adaptive_eig_tol && std::isfinite(prevD)) ek.tol = std::max(eo.tol, std::min(1e-3, 0.1 * prevD));
        // the first iteration of the atomic start begins from the atomic orbitals (or, with
        // none, from the reference's seeds); later ones from the previous orbitals
        const bool first_atoms = atoms_start && it == 1;
        const double* sb = first_atoms && nao > 0 ? aobuf.p : nullptr;
        rec.eig_iterations_alpha = solve_orbitals(ctx, g, va.p, nconv_a, bands_a, psia.p, ld, !first_atoms,
                                                  eiga.data(), resa.data(), ek, sb, nao);
        if (!closed)
            rec.eig_iterations_beta = solve_orbitals(ctx, g, vb.p, nconv_b, bands_b, psib.p, ld, !first_atoms,
                                                     eigb.data(), resb.data(), ek, sb, nao);
        if (first_atoms && aobuf.p) aobuf.release();
        if (kt > 0.0) {
            nconv_a = fermi(eiga, na, occa);
            if (closed) {
                occb = occa;
                nconv_b = nconv_a;
            } else {
                nconv_b = fermi(eigb, nb, occb);
            }
        }
        rec.ms_orbitals = ms_since(t0);
        // output densities (:160-187)
        t0 = Clock::now();
        spin_density(ctx, N, psia.p, bands_a, ld, occa.data(), oa.p);
        if (closed) DFT_CUDA(cudaMemcpyAsync(ob.p, oa.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
        else spin_density(ctx, N, psib.p, bands_b, ld, occb.data(), ob.p);
        add2(ctx, N, oa.p, ob.p, orho.p);
        if (vpredict_out && it > 1) {
            add_into(ctx, N, vh.p, vres.p, ovh.p);
            if (monopole) sub(ctx, N, ovh.p, mvc.p, mvp1.p);
        }
        JacobiResult jout = poisson(orho.p, ovh.p, it > 1);
        if (vpredict_out) sub(ctx, N, ovh.p, vh.p, vres.p);
        sync(ctx);
        rec.ms_density = ms_since(t0);
        rec.poisson_sweeps_out = jout.sweeps;
        rec.poisson_cycles_out = last_cycles;
        // energies (TotalEnergyMolecule.cpp:237-333): orbitals alpha then beta in one sum
        t0 = Clock::now();
        double T = 0.0;
        if (kt > 0.0) {
            // fractional occupations over every band that carries charge
            kinetic_per_band(ctx, g, psia.p, nconv_a, ld, Ta.data());
            if (!closed) kinetic_per_band(ctx, g, psib.p, nconv_b, ld, Tb.data());
            for (int i = 0; i < nconv_a; ++i) T += occa[i] * Ta[i];
            for (int i = 0; i < (closed ? nconv_a : nconv_b); ++i) T += occb[i] * (closed ? Ta[i] : Tb[i]);
        } else {
            kinetic_per_band(ctx, g, psia.p, na, ld, Ta.data());
            if (!closed) kinetic_per_band(ctx, g, psib.p, nb, ld, Tb.data());
            for (int i = 0; i < na; ++i) T += 1.0 * Ta[i];
            for (int i = 0; i < nb; ++i) T += 1.0 * (closed ? Ta[i] : Tb[i]);
        }
        const double eext = dot3(ctx, N, orho.p, vext.p, g.dV);
        const double eh = 0.5 * dot(ctx, N, orho.p, ovh.p) * g.dV;
        const double exc = xc(ctx, g, kind, oa.p, ob.p, nullptr, nullptr, true);
        E[0] = T;
        E[1] = eext;
        E[2] = eh;
        E[3] = exc;
        E[4] = enn;
        E[5] = T + eext + eh + exc + enn;
        // convergence measures (:201-250, MolecularSCFHelpers.cpp:46-183)
        const double dd = density_difference(ctx, g, rho.p, orho.p);
        const double sdd = std::max(density_difference(ctx, g, da.p, oa.p), density_difference(ctx, g, db.p, ob.p));
        effd = std::max(dd, sdd);
        resid = 0.0;
        for (int i = 0; i < na; ++i) resid = std::max(resid, resa[i]);
        if (!closed)
            for (int i = 0; i < nb; ++i) resid = std::max(resid, resb[i]);
        rec.ms_energy = ms_since(t0);
        dE = std::isfinite(prevE) ? std::fabs(E[5] - prevE) : std::numeric_limits<double>::infinity();
        // occupied eigenvalues (alpha, then beta) and their change since the previous iteration
        {
            std::vector<double> cur(eiga.begin(), eiga.begin() + na);
            const std::vector<double>& eb = closed ? eiga : eigb;
            cur.insert(cur.end(), eb.begin(), eb.begin() + nb);
            deig = std::numeric_limits<double>::infinity();
            if (prev_eig.size() == cur.size()) {
                deig = 0.0;
                for (size_t q = 0; q < cur.size(); ++q) deig = std::max(deig, std::fabs(cur[q] - prev_eig[q]));
            }
            prev_eig.swap(cur);
        }
        rec.eigenvalue_difference = deig;
        converged = dE < o.energy_tol && effd < o.density_tol && resid < o.ks_tol;
        rec.energy = E[5];
        rec.energy_difference = dE;
        rec.density_difference = effd;
        rec.ks_residual = resid;
        rec.mixing = o.mixer == 1 ? pbeta : imix;
        rec.ms_total = ms_since(t_it);
        if (res->history && res->history_len < res->history_capacity) res->history[res->history_len++] = rec;
        if (dE < o.energy_tol) res->last_energy_criterion_iteration = it;
        if (effd < o.density_tol) res->last_density_criterion_iteration = it;
        if (resid < o.ks_tol) res->last_ks_criterion_iteration = it;
        res->min_energy_difference = std::min(res->min_energy_difference, dE);
        res->min_density_difference = std::min(res->min_density_difference, effd);
        res->min_ks_residual = std::min(res->min_ks_residual, resid);
        res->final_mixing = rec.mixing;
        if (log) {
            std::fprintf(log,
                         "{\"iteration\":%d,\"energy\":%s,\"energy_difference\":%s,\"density_difference\":%s,"
                         "\"ks_residual\":%s,\"mixing\":%s,\"kinetic\":%s,\"external\":%s,\"hartree\":%s,"
                         "\"exchange_correlation\":%s,\"nuclear_repulsion\":%s,\"poisson_sweeps_in\":%ld,"
                         "\"poisson_sweeps_out\":%ld,\"poisson_cycles_in\":%d,\"poisson_cycles_out\":%d,"
                         "\"eig_iterations_alpha\":%d,\"eig_iterations_beta\":%d,\"eigenvalue_difference\":%s,\"levels_alpha\":%s,\"levels_beta\":%s,\"ms_hartree\":%s,\"ms_xc\":%s,"
                         "\"ms_orbitals\":%s,\"ms_density\":%s,\"ms_energy\":%s,\"ms_total\":%s}\n",
                         it, jnum(E[5]).c_str(), jnum(dE).c_str(), jnum(effd).c_str(), jnum(resid).c_str(),
                         jnum(rec.mixing).c_str(), jnum(E[0]).c_str(), jnum(E[1]).c_str(), jnum(E[2]).c_str(),
                         jnum(E[3]).c_str(), jnum(E[4]).c_str(), jin.sweeps, jout.sweeps, rec.poisson_cycles_in,
                         rec.poisson_cycles_out, rec.eig_iterations_alpha,
                         rec.eig_iterations_beta, jnum(deig).c_str(), jlevels(eiga, na).c_str(),
                         jlevels(closed ? eiga : eigb, nb).c_str(), jnum(rec.ms_hartree).c_str(),
                         jnum(rec.ms_xc).c_str(), jnum(rec.ms_orbitals).c_str(), jnum(rec.ms_density).c_str(),
                         jnum(rec.ms_energy).c_str(), jnum(rec.ms_total).c_str());
            std::fflush(log);
        }
        if (o.verbose)
            fprintf(stderr,
                    "[scf] it=%3d E=%.12f dE=%.3e dRho=%.3e KS=%.3e mix=%.3f sweeps=%ld/%ld eig_it=%d/%d  %.1f ms\n", it,
                    E[5], dE, effd, resid, imix, jin.sweeps, jout.sweeps, rec.eig_iterations_alpha,
                    rec.eig_iterations_beta, rec.ms_total);
        if (o.verbose > 1) {
            // per spin: the lowest levels, the levels around the highest occupied one, and the
            // spin density change, to tell level crossings at the Fermi level from sloshing
            auto levels = [&](const char* tag, const std::vector<double>& e, int nocc, double dr) {
                const int m = (int)e.size();
                fprintf(stderr, "[scf]   %s dRho=%.3e low:", tag, dr);
                for (int i = 0; i < std::min(3, m); ++i) fprintf(stderr, " %.5f", e[i]);
                fprintf(stderr, " | homo-3..:");
                for (int i = std::max(0, nocc - 4); i < std::min(m, nocc + 4); ++i)
                    fprintf(stderr, "%s%.5f", i == nocc ? " || " : " ", e[i]);
                fprintf(stderr, "\n");
            };
            levels("a", eiga, na, density_difference(ctx, g, da.p, oa.p));
            if (!closed) levels("b", eigb, nb, density_difference(ctx, g, db.p, ob.p));
            if (o.verbose > 2) {
                // where the levels around the Fermi level live: fraction within 4 bohr of a face
                fprintf(stderr, "[scf]   wall fraction (4 bohr) alpha homo-3..:");
                for (int i = std::max(0, na - 4); i < std::min(bands_a, na + 4); ++i)
                    fprintf(stderr, "%s%.3f", i == na ? " || " : " ", wall_fraction(ctx, g, psia.p + (long long)i * ld, 4.0));
                fprintf(stderr, "\n");
            }
        }
        if (converged) break;
        if (o.stop_abs_de > 0.0 && dE < o.stop_abs_de && (o.stop_abs_deig <= 0.0 || deig < o.stop_abs_deig) &&
            (o.stop_abs_drho <= 0.0 || effd < o.stop_abs_drho))
            break;
        // adaptive mixing with the pre-update factor applied (:447-484)
        if (std::isfinite(prevD)) {
            if (effd > prevD * 1.05) mixing = std::max(0.10, mixing * 0.75);
            else if (effd < prevD) mixing = std::min(0.50, mixing * 1.10);
        }
        if (o.mixer == 1) {
            pulay_mix();
        } else if (kq0 > 0.0) {
            // n_in += mixing * K(n_out - n_in)
            sub(ctx, N, oa.p, da.p, kbuf.p);
            if (!closed) sub(ctx, N, ob.p, db.p, kbuf.p + N);
            double* dst[2] = {da.p, db.p};
            const double* rr[2] = {kbuf.p, kbuf.p + N};
            kerker_update(ctx, g, ns, dst, rr, kbuf.p + (size_t)ns * N, kbuf.p + (size_t)(ns + 1) * N, kq2, imix);
            if (closed)
                DFT_CUDA(cudaMemcpyAsync(db.p, da.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, ctx->stream));
        } else {
            mix(ctx, N, da.p, oa.p, imix);
            mix(ctx, N, db.p, ob.p, imix);
        }
        if (vpredict && o.mixer == 0) mix(ctx, N, vh.p, ovh.p, imix);  // V_in + m (V_out - V_in)
        if (vpredict && monopole) sub(ctx, N, vh.p, mvc.p, mvp0.p);   // the zero-face part's start
        prevD = effd;
        prevE = E[5];
    }
    // (skipped when the caller's own Jacobi stop is already that tight: a target below 1e-13
    // is rounding noise and would only run the sweep cap)
    if (pstart == DFT_POISSON_MULTIGRID && it >= 1 && o.poisson_tol * fixed_scale >= 1e-13) {
        // The reported Hartree energy enters the total at first order in the error of
        // V_H(n_out): with multigrid starts the last V_H(n_out) is taken on to the Jacobi fixed
        // point (the max|dV| rule scaled by 1 - rho_Jacobi, a few cycles from the potential at
        // hand) before E_H and E_tot are reported.  The density is unchanged.
        poisson(orho.p, ovh.p, true, o.poisson_tol * fixed_scale);
        const double eh = 0.5 * dot(ctx, N, orho.p, ovh.p) * g.dV;
        E[5] += eh - E[2];
        E[2] = eh;
    }
    sync(ctx);
    res->kinetic = E[0];
    res->external = E[1];
    res->hartree = E[2];
    res->exchange_correlation = E[3];
    res->nuclear_repulsion = E[4];
    res->total = E[5];
    res->iterations = std::min(it, o.max_iterations);
    res->converged = converged ? 1 : 0;
    res->density_difference = effd;
    res->energy_difference = dE;
    res->max_ks_residual = resid;
    res->n_alpha = na;
    res->n_beta = nb;
    if (res->eigenvalues) {
        for (int i = 0; i < na; ++i) res->eigenvalues[i] = eiga[i];
        for (int i = 0; i < nb; ++i) res->eigenvalues[na + i] = closed ? eiga[i] : eigb[i];
    }
    if (res->alpha_density)
        DFT_CUDA(cudaMemcpyAsync(res->alpha_density, oa.p, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->stream));
    if (res->beta_density)
        DFT_CUDA(cudaMemcpyAsync(res->beta_density, ob.p, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->stream));
    if (res->alpha_potential)
        DFT_CUDA(cudaMemcpyAsync(res->alpha_potential, va.p, sizeof(double) * N, cudaMemcpyDeviceToHost, ctx->stream));
    if (res->beta_potential)
        DFT_CUDA(cudaMemcpyAsync(res->beta_potential, closed ? va.p : vb.p, sizeof(double) * N, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    if (res->orbitals) {
        DFT_CUDA(cudaMemcpyAsync(res->orbitals, psia.p, sizeof(double) * N * na, cudaMemcpyDeviceToHost, ctx->stream));
        DFT_CUDA(cudaMemcpyAsync(res->orbitals + (size_t)na * N, closed ? psia.p : psib.p, sizeof(double) * N * nb,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    }
    sync(ctx);
    res->seconds = ms_since(t_start) * 1e-3;
    if (log) {
        std::fprintf(log,
                     "{\"result\":{\"electrons\":%d,\"charge\":%d,\"multiplicity\":%d,\"converged\":%s,"
                     "\"iterations\":%d,\"energy\":{\"kinetic\":%s,\"external\":%s,\"hartree\":%s,"
                     "\"exchangeCorrelation\":%s,\"nuclearRepulsion\":%s,\"total\":%s},"
                     "\"densityDifference\":%s,\"energyDifference\":%s,\"maxKSResidual\":%s,"
                     "\"convergenceAnalysis\":{\"lastEnergyCriterionIteration\":%d,"
                     "\"lastDensityCriterionIteration\":%d,\"lastKSCriterionIteration\":%d,"
                     "\"minimumEnergyDifference\":%s,\"minimumDensityDifference\":%s,\"minimumKSResidual\":%s,"
                     "\"finalMixing\":%s},\"alphaLevels\":%s,\"betaLevels\":%s,\"seconds\":%s}}\n",
                     ne, charge, multiplicity, converged ? "true" : "false", res->iterations, jnum(E[0]).c_str(),
                     jnum(E[1]).c_str(), jnum(E[2]).c_str(), jnum(E[3]).c_str(), jnum(E[4]).c_str(),
                     jnum(E[5]).c_str(), jnum(effd).c_str(), jnum(dE).c_str(), jnum(resid).c_str(),
                     res->last_energy_criterion_iteration, res->last_density_criterion_iteration,
                     res->last_ks_criterion_iteration, jnum(res->min_energy_difference).c_str(),
                     jnum(res->min_density_difference).c_str(), jnum(res->min_ks_residual).c_str(),
                     jnum(res->final_mixing).c_str(), jlevels(eiga, na).c_str(),
                     jlevels(closed ? eiga : eigb, nb).c_str(), jnum(res->seconds).c_str());
    }
}

}  // namespace dftb
