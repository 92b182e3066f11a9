// Superposition-of-atoms start for the molecular SCF.
//
// The reference starts the molecular SCF from orbitals of the bare nuclear potential
// (buildInitialMolecularDensities, MolecularSCFHelpers.cpp:515-579): a full Davidson solve
// in V_ext whose density is far from the self-consistent one.  This option starts instead
// from the converged radial atoms of the same functional (solveSelfConsistentField,
// SelfConsistentField.cpp:539-786, batched on the device by radial.cu): their spherical
// densities summed at every grid node, and one start vector per occupied atomic orbital for
// the first eigensolve.  The SCF's stop tests are unchanged, so only the path to the fixed
// point differs.
#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "ops.h"

namespace dftb {

namespace {

constexpr long RADIAL_POINTS = 2000;  // the reference's radial grid (RadialGrid(2000, 30))
constexpr double RADIAL_RMAX = 30.0;

struct AtomSite {
    double x, y, z;
    int table;  // row of the radial tables
};

// f(r) by linear interpolation on r_i = (i + 1) hr (RadialGrid.cpp:16-20); f(r_0) below r_0,
// zero beyond the last node
__device__ __forceinline__ double radial_interp(const double* __restrict__ f, int npts, double hr, double r) {
    const double u = r / hr - 1.0;
    if (u <= 0.0) return f[0];
    const int i = (int)u;
    if (i >= npts - 1) return 0.0;
    const double t = u - (double)i;
    return (1.0 - t) * f[i] + t * f[i + 1];
}

// out[p] = sum_a n_{Z_a}(|x_p - R_a|); per-block partial sums of out for the normalisation
__global__ void __launch_bounds__(256) superpose_kernel(Grid g, int nsite, const AtomSite* __restrict__ sites,
                                                        const double* __restrict__ dens, int npts, double hr,
                                                        double* __restrict__ out, double* __restrict__ partial) {
    __shared__ double sh[8];
    double acc = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const double x = g.xmin + i * g.dx, y = g.ymin + j * g.dy, z = g.zmin + k * g.dz;
        double s = 0.0;
        for (int a = 0; a < nsite; ++a) {
            const double dx = x - sites[a].x, dy = y - sites[a].y, dz = z - sites[a].z;
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            s += radial_interp(dens + (long long)sites[a].table * npts, npts, hr, r);
        }
        out[p] = s;
        acc += s;
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// da = c_a n, db = c_b n (db may be null)
__global__ void split_kernel(long long n, const double* __restrict__ tot, double ca, double cb, double* __restrict__ da,
                             double* __restrict__ db) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double v = tot[p];
        da[p] = ca * v;
        if (db) db[p] = cb * v;
    }
}

struct AOFunc {
    int site, shell, l, m;
};

// One atomic-orbital start vector per blockIdx.y: u_nl(r)/r times the real angular factor
// (s: 1; p: x/r, y/r, z/r; d: xy, xz, yz, x^2 - y^2, 3z^2 - r^2 over r^2).
__global__ void ao_basis_kernel(Grid g, const AOFunc* __restrict__ funcs, const AtomSite* __restrict__ sites,
                                const double* __restrict__ orbs, int npts, double hr, int max_shells,
                                double* __restrict__ basis, long long ld) {
    const AOFunc f = funcs[blockIdx.y];
    const AtomSite s = sites[f.site];
    const double* u = orbs + ((long long)s.table * max_shells + f.shell) * npts;
    const double r0 = hr;
    double* out = basis + (long long)blockIdx.y * ld;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const double dx = g.xmin + i * g.dx - s.x, dy = g.ymin + j * g.dy - s.y, dz = g.zmin + k * g.dz - s.z;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double R = radial_interp(u, npts, hr, r) / fmax(r, r0);
        double ang = 1.0;
        if (f.l > 0) {
            if (r < 1e-12) {
                ang = 0.0;
            } else if (f.l == 1) {
                ang = (f.m == 0 ? dx : f.m == 1 ? dy : dz) / r;
            } else {
                const double r2 = r * r;
                switch (f.m) {
                    case 0: ang = dx * dy / r2; break;
                    case 1: ang = dx * dz / r2; break;
                    case 2: ang = dy * dz / r2; break;
                    case 3: ang = (dx * dx - dy * dy) / r2; break;
                    default: ang = (3.0 * dz * dz - r2) / r2; break;
                }
            }
        }
        out[p] = R * ang;
    }
}

}  // namespace

int atomic_start(dft_context* ctx, const Grid& g, int nnuc, const int* Z, const double* xyz, int kind, int ne_a,
                 int ne_b, double* da, double* db, double* basis, long long ld, int max_basis) {
    if (nnuc <= 0) fail(DFT_INVALID_ARGUMENT, "no nuclei");
    // one radial run per element
    std::map<int, int> table;
    std::vector<int> elems;
    for (int a = 0; a < nnuc; ++a) {
        if (Z[a] < 1 || Z[a] > 30) fail(DFT_INVALID_ARGUMENT, "the atomic start has atoms Z = 1..30 only (Z = %d)", Z[a]);
        if (!table.count(Z[a])) {
            table[Z[a]] = (int)elems.size();
            elems.push_back(Z[a]);
        }
    }
    const int nz = (int)elems.size();
    const size_t dens_n = (size_t)nz * RADIAL_POINTS, orbs_n = (size_t)nz * RADIAL_MAX_SHELLS * RADIAL_POINTS;
    std::vector<AtomSite> sites(nnuc);
    for (int a = 0; a < nnuc; ++a) sites[a] = {xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2], table[Z[a]]};
    const int nblk = std::max(1, std::min((int)((g.N + 255) / 256), ctx->num_sms * 4));
    // one slab: radial tables, sites, basis functions, partial sums
    const size_t site_b = sizeof(AtomSite) * nnuc, func_cap = (size_t)nnuc * 16;
    const size_t bytes = sizeof(double) * (dens_n + orbs_n + nblk + 8) + site_b + sizeof(AOFunc) * func_cap + 256;
    char* slab = (char*)ws_get(ctx, WS_TMP3, bytes);
    double* dens = (double*)slab;
    double* orbs = dens + dens_n;
    double* partial = orbs + orbs_n;
    AtomSite* dsites = (AtomSite*)(partial + nblk + 8);
    AOFunc* dfuncs = (AOFunc*)((char*)dsites + ((site_b + 15) / 16) * 16);
    std::vector<std::vector<std::array<int, 2>>> shells;
    radial_atom_tables(ctx, nz, elems.data(), kind, RADIAL_POINTS, RADIAL_RMAX, dens, orbs, shells);
    DFT_CUDA(cudaMemcpyAsync(dsites, sites.data(), site_b, cudaMemcpyHostToDevice, ctx->stream));
    const double hr = RADIAL_RMAX / (double)(RADIAL_POINTS + 1);
    // total density at the nodes, its sum, then the split by spin scaled to the electron counts
    double* tot = da;
    superpose_kernel<<<nblk, 256, 0, ctx->stream>>>(g, nnuc, dsites, dens, (int)RADIAL_POINTS, hr, tot, partial);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    double* hp = pinned(ctx, nblk);
    DFT_CUDA(cudaMemcpyAsync(hp, partial, sizeof(double) * nblk, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    double sum = 0.0;
    for (int b = 0; b < nblk; ++b) sum += hp[b];
    const double count = sum * g.dV;
    if (!(count > 0.0) || !std::isfinite(count)) fail(DFT_NUMERICAL, "superposed atomic density is empty on this grid");
    split_kernel<<<nblk, 256, 0, ctx->stream>>>(g.N, tot, ne_a / count, ne_b / count, da, db);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    if (!basis || max_basis <= 0) return 0;
    // start vectors: every occupied alpha shell of every atom, 2l + 1 real functions each
    std::vector<AOFunc> funcs;
    for (int a = 0; a < nnuc; ++a) {
        const auto& sh = shells[table[Z[a]]];
        for (int k = 0; k < (int)sh.size(); ++k) {
            const int l = sh[k][1];
            if (l > 2) continue;
            for (int m = 0; m < 2 * l + 1; ++m)
                if ((int)funcs.size() < std::min<int>(max_basis, (int)func_cap)) funcs.push_back({a, k, l, m});
        }
    }
    const int nf = (int)funcs.size();
    if (nf == 0) return 0;
    DFT_CUDA(cudaMemcpyAsync(dfuncs, funcs.data(), sizeof(AOFunc) * nf, cudaMemcpyHostToDevice, ctx->stream));
    const int bx = std::max(1, std::min((int)((g.N + 255) / 256), std::max(1, ctx->num_sms * 8 / nf)));
    ao_basis_kernel<<<dim3(bx, nf), 256, 0, ctx->stream>>>(g, dfuncs, dsites, orbs, (int)RADIAL_POINTS, hr,
                                                           RADIAL_MAX_SHELLS, basis, ld);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    sync(ctx);
    return nf;
}

}  // namespace dftb
