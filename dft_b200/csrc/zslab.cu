// Z-slab domain decomposition of the 3D grid: the pieces one rank runs on its own slab.
//
// A slab holds the global planes [z_lo, z_hi) of the x-fastest layout, i.e. its own planes
// plus halo planes copied from the neighbouring slabs.  The host driver (dft_b200/zslab.py)
// exchanges the halos and reduces the stop measures over ranks; nothing here waits on another
// rank or another kernel.
//
// Jacobi (reference HartreePotentialMolecule.cpp:207-321): a slab with T halo planes on each
// side can run T sweeps between exchanges.  Every sweep updates all interior planes of the
// slab; the outermost planes stay fixed, so after s <= T sweeps the planes at distance >= s
// from the slab's edges -- every owned plane -- hold exactly the values of the single-domain
// solve.  The stop measure max|V' - V| is folded only over owned planes and kept per sweep, so
// the driver can reduce it over ranks and find the sweep at which the single-domain loop stops.
// A block of sweeps reads its start and never writes it (the result goes to a second buffer,
// through a third), so a block that overshoots the stop is replayed from the untouched start
// without a snapshot copy.  Same arithmetic and operation order as jacobi_sweep_kernel:
// bit-identical values.
//
// H psi (reference KohnShamHamiltonianMolecule.cpp:78-177): with one halo plane per side the
// owned planes of a slab see the same six neighbours as on the whole grid, and the grid's own
// faces (where no neighbour exists) are slab faces too, so apply_hamiltonian on the slab's
// plane count gives bit-identical owned planes.
//
// XC (reference ExchangeCorrelationMolecule.cpp:576-842): the potential at a plane needs the
// gradient coefficients one plane away, which need the densities two planes away, so with two
// halo planes per side the XC kernels on the slab give bit-identical owned planes.  The energy
// is summed over the owned planes only; ranks add their parts.
//
// Gram products: the sum over points splits into per-rank sums over owned planes.
#include <algorithm>
#include <cmath>

#include "ops.h"
#include "xc_device.cuh"
#include "xc_grad.cuh"

namespace dftb {
namespace {

constexpr int SB_X = 32, SB_Y = 8;

// Slab initial state: face values of the global grid (the reference's boundary rule,
// HartreePotentialMolecule.cpp:37-95, as in jacobi_init_kernel) on the slab's part of the six
// faces; the interior is 0 (cold start) or the interior of `guess` (same slab layout).
__global__ void slab_init_kernel(Grid g, int z_lo, long long n_local, double Q, double* __restrict__ v,
                                 const double* __restrict__ guess) {
    const long long sxy = (long long)g.nx * g.ny;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n_local;
         p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx);
        const int j = (int)((p / g.nx) % g.ny);
        const int k = z_lo + (int)(p / sxy);
        const bool face = i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz;
        double val = 0.0;
        if (!face && guess) val = guess[p];
        if (face) {
            const double x = __dadd_rn(g.xmin, __dmul_rn((double)i, g.dx));
            const double y = __dadd_rn(g.ymin, __dmul_rn((double)j, g.dy));
            const double z = __dadd_rn(g.zmin, __dmul_rn((double)k, g.dz));
            const double d[6] = {fabs(x - g.xmin), fabs(x - g.xmax), fabs(y - g.ymin),
                                 fabs(y - g.ymax), fabs(z - g.zmin), fabs(z - g.zmax)};
            double m2 = INFINITY;
            for (int q = 0; q < 6; ++q) m2 = fmin(m2, __dmul_rn(d[q], d[q]));
            if (m2 > 0.0) {
                const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
                if (r > 0.0) val = Q / r;
            }
        }
        v[p] = val;
    }
}

// One Jacobi sweep over the slab's interior planes 1..nzl-2 (local indices), x and y interior
// as on the whole grid.  max|V' - V| over the local planes [own_lo, own_hi) goes into
// *diff_bits (a non-negative double orders like its bit pattern, so atomicMax on the bits is
// the maximum; the caller zeroes the word).
__global__ void __launch_bounds__(SB_X* SB_Y) slab_sweep_kernel(int nx, int ny, int nzl, double ix2, double iy2,
                                                                double iz2, double den,
                                                                const double* __restrict__ rho,
                                                                const double* __restrict__ cur,
                                                                double* __restrict__ nxt, int own_lo, int own_hi,
                                                                int zchunk, unsigned long long* diff_bits) {
    __shared__ double sh[SB_X * SB_Y / 32];
    const double c4pi = 4.0 * xcf::PI;
    const int i = blockIdx.x * SB_X + threadIdx.x;
    const int j = blockIdx.y * SB_Y + threadIdx.y;
    double md = 0.0;
    if (i >= 1 && i + 1 < nx && j >= 1 && j + 1 < ny) {
        const int sxy = nx * ny;
        const int kb = max(1, (int)blockIdx.z * zchunk);
        const int ke = min(nzl - 1, (int)(blockIdx.z + 1) * zchunk);
        if (kb < ke) {
            int idx = kb * sxy + j * nx + i;
            double below = __ldg(cur + idx - sxy);
            double c = __ldg(cur + idx);
#pragma unroll 4
            for (int k = kb; k < ke; ++k, idx += sxy) {
                const double above = __ldg(cur + idx + sxy);
                const double sx = __dadd_rn(__ldg(cur + idx - 1), __ldg(cur + idx + 1));
                const double sy = __dadd_rn(__ldg(cur + idx - nx), __ldg(cur + idx + nx));
                const double sz = __dadd_rn(below, above);
                double acc = __dadd_rn(__dmul_rn(ix2, sx), __dmul_rn(iy2, sy));
                acc = __dadd_rn(acc, __dmul_rn(iz2, sz));
                acc = __dadd_rn(acc, __dmul_rn(c4pi, __ldg(rho + idx)));
                const double v = __ddiv_rn(acc, den);
                nxt[idx] = v;
                if (k >= own_lo && k < own_hi) md = fmax(md, fabs(v - c));
                below = c;
                c = above;
            }
        }
    }
    const int tid = threadIdx.y * SB_X + threadIdx.x;
    md = warp_max(md);
    if ((tid & 31) == 0) sh[tid >> 5] = md;
    __syncthreads();
    if (tid == 0) {
        double m = sh[0];
        for (int w = 1; w < SB_X * SB_Y / 32; ++w) m = fmax(m, sh[w]);
        if (m > 0.0) atomicMax(diff_bits, (unsigned long long)__double_as_longlong(m));
    }
}

// Copies the points a sweep never writes -- the first and last plane of the slab and the x/y
// faces of the planes between -- from src to both destinations (the shell, enumerated directly:
// 2 nx ny + 2 nx (nzl-2) + 2 (ny-2) (nzl-2) points).  Needs nx, ny, nzl >= 3.
__global__ void slab_shell_copy_kernel(int nx, int ny, int nzl, const double* __restrict__ src,
                                       double* __restrict__ d0, double* __restrict__ d1) {
    const long long sxy = (long long)nx * ny;
    const long long nA = 2 * sxy;                          // planes 0 and nzl-1
    const long long nB = 2LL * nx * (nzl - 2);             // rows j = 0, ny-1 of planes 1..nzl-2
    const long long nC = 2LL * (ny - 2) * (nzl - 2);       // columns i = 0, nx-1 of rows 1..ny-2
    const long long total = nA + nB + nC;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        long long p;
        if (q < nA) {
            p = q < sxy ? q : (long long)(nzl - 1) * sxy + (q - sxy);
        } else if (q < nA + nB) {
            const long long r = q - nA;
            const long long k = 1 + r / (2LL * nx), rem = r % (2LL * nx);
            const long long j = rem < nx ? 0 : ny - 1, i = rem < nx ? rem : rem - nx;
            p = k * sxy + j * nx + i;
        } else {
            const long long r = q - nA - nB;
            const long long k = 1 + r / (2LL * (ny - 2)), rem = r % (2LL * (ny - 2));
            const long long j = 1 + (rem < ny - 2 ? rem : rem - (ny - 2)), i = rem < ny - 2 ? 0 : nx - 1;
            p = k * sxy + j * nx + i;
        }
        const double v = src[p];
        d0[p] = v;
        d1[p] = v;
    }
}

// Sum of n eps dV over the points [p_lo, p_hi) of a slab (one partial per block), gradients
// from the whole slab as in xc_point_kernel.
template <int KIND>
__global__ void __launch_bounds__(256) slab_xc_energy_kernel(Grid s, long long p_lo, long long p_hi,
                                                             const double* __restrict__ na,
                                                             const double* __restrict__ nb,
                                                             double* __restrict__ partial) {
    __shared__ double sh[8];
    double e = 0.0;
    for (long long p = p_lo + (long long)blockIdx.x * blockDim.x + threadIdx.x; p < p_hi;
         p += (long long)gridDim.x * blockDim.x) {
        const double a = na[p], b = nb[p];
        const double n = a + b;
        if (n > xcf::RHO_FLOOR) {
            const int i = (int)(p % s.nx);
            const int j = (int)((p / s.nx) % s.ny);
            const int k = (int)(p / ((long long)s.nx * s.ny));
            double ga = 0.0, gb = 0.0;
            if (KIND == 1) {
                ga = gradmag(s, na, p, i, j, k);
                gb = gradmag(s, nb, p, i, j, k);
            }
            e += n * xcf::evaluate<KIND>(a, b, ga, gb).eps * s.dV;
        }
    }
    e = block_sum(e, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = e;
}

// The slab as a Grid: the global spacing and bounds (so every constant is the whole grid's),
// the slab's plane count.
Grid slab_grid(const Grid& g, int z_lo, int z_hi) {
    Grid s = g;
    s.nz = z_hi - z_lo;
    s.N = (long long)g.nx * g.ny * s.nz;
    return s;
}

void check_slab(const Grid& g, int z_lo, int z_hi) {
    if (z_lo < 0 || z_hi > g.nz || z_hi <= z_lo) fail(DFT_INVALID_ARGUMENT, "slab planes must satisfy 0 <= z_lo < z_hi <= nz");
}

}  // namespace

void zslab_jacobi_init(dft_context* ctx, const Grid& g, int z_lo, int z_hi, double Q, const double* guess, double* v) {
    check_slab(g, z_lo, z_hi);
    const long long n = (long long)g.nx * g.ny * (z_hi - z_lo);
    const int blocks = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)ctx->num_sms * 8));
    slab_init_kernel<<<blocks, 256, 0, ctx->stream>>>(g, z_lo, n, Q, v, guess);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void zslab_jacobi_sweeps(dft_context* ctx, const Grid& g, int z_lo, int z_hi, int own_lo, int own_hi,
                         const double* rho, const double* v_in, double* v_out, double* scratch, int sweeps,
                         double* diffs) {
    check_slab(g, z_lo, z_hi);
    if (own_lo > own_hi || own_lo < z_lo || own_hi > z_hi)
        fail(DFT_INVALID_ARGUMENT, "owned planes must lie inside the slab");
    // an owned plane that the whole grid updates must be one the slab updates
    if ((own_lo < own_hi) && ((own_lo < z_lo + 1 && own_lo != 0) || (own_hi > z_hi - 1 && own_hi != g.nz)))
        fail(DFT_INVALID_ARGUMENT, "an owned interior plane lies on the slab's edge (no halo plane beyond it)");
    if (sweeps < 0) fail(DFT_INVALID_ARGUMENT, "sweeps must be >= 0");
    const Grid s = slab_grid(g, z_lo, z_hi);
    if (sweeps > 0) DFT_CUDA(cudaMemsetAsync(diffs, 0, sizeof(double) * (size_t)sweeps, ctx->stream));
    if (sweeps == 0 || s.nx < 3 || s.ny < 3 || s.nz < 3) {
        // nothing to update: the state after the sweeps is the start (every diff stays 0)
        DFT_CUDA(cudaMemcpyAsync(v_out, v_in, sizeof(double) * (size_t)s.N, cudaMemcpyDeviceToDevice, ctx->stream));
        return;
    }
    {
        const long long shell = 2LL * s.nx * s.ny + 2LL * s.nx * (s.nz - 2) + 2LL * (s.ny - 2) * (s.nz - 2);
        const int blocks = (int)std::min<long long>((shell + 255) / 256, (long long)ctx->num_sms * 4);
        slab_shell_copy_kernel<<<blocks, 256, 0, ctx->stream>>>(s.nx, s.ny, s.nz, v_in, v_out, scratch);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    const int bx = (s.nx + SB_X - 1) / SB_X, by = (s.ny + SB_Y - 1) / SB_Y;
    int zc = 32;
    while (zc > 4 && (long long)bx * by * ((s.nz + zc - 1) / zc) < 2LL * ctx->num_sms) zc >>= 1;
    const dim3 grid(bx, by, (s.nz + zc - 1) / zc), block(SB_X, SB_Y);
    const int lo = own_lo - z_lo, hi = own_hi - z_lo;
    unsigned long long* bits = reinterpret_cast<unsigned long long*>(diffs);
    // sweep t writes v_out when sweeps - 1 - t is even, so the last one lands there; v_in is
    // only read
    const double* cur = v_in;
    for (int t = 0; t < sweeps; ++t) {
        double* nxt = ((sweeps - 1 - t) & 1) ? scratch : v_out;
        slab_sweep_kernel<<<grid, block, 0, ctx->stream>>>(s.nx, s.ny, s.nz, g.ix2, g.iy2, g.iz2, den, rho, cur, nxt,
                                                           lo, hi, zc, bits + t);
        cur = nxt;
    }
    DFT_LAUNCH_CHECK();
    count_launch(ctx, sweeps);
}

void zslab_hamiltonian(dft_context* ctx, const Grid& g, int z_lo, int z_hi, const double* V, const double* psi,
                       double* hpsi, int nbands, long long ld) {
    check_slab(g, z_lo, z_hi);
    const Grid s = slab_grid(g, z_lo, z_hi);
    if (ld < s.N) fail(DFT_INVALID_ARGUMENT, "ld must be >= nx*ny*(z_hi - z_lo)");
    apply_hamiltonian(ctx, s, V, psi, hpsi, nbands, ld);
}

double zslab_xc(dft_context* ctx, const Grid& g, int z_lo, int z_hi, int own_lo, int own_hi, int kind,
                const double* na, const double* nb, double* va, double* vb) {
    check_slab(g, z_lo, z_hi);
    if (own_lo > own_hi || own_lo < z_lo || own_hi > z_hi)
        fail(DFT_INVALID_ARGUMENT, "owned planes must lie inside the slab");
    // two planes beyond the owned ones on each side, unless the slab ends at a face of g
    if (own_lo < own_hi && ((z_lo > 0 && own_lo - z_lo < 2) || (z_hi < g.nz && z_hi - own_hi < 2)))
        fail(DFT_INVALID_ARGUMENT, "XC on a slab needs two halo planes beyond the owned planes");
    if (kind != DFT_XC_PZ81 && kind != DFT_XC_PBE96) fail(DFT_INVALID_ARGUMENT, "unknown functional kind %d", kind);
    const Grid s = slab_grid(g, z_lo, z_hi);
    if (va || vb) xc(ctx, s, kind, na, nb, va, vb, false);
    const long long sxy = (long long)s.nx * s.ny;
    const long long p_lo = (long long)(own_lo - z_lo) * sxy, p_hi = (long long)(own_hi - z_lo) * sxy;
    if (p_hi <= p_lo) return 0.0;
    const int nbk = (int)std::max<long long>(1, std::min<long long>((p_hi - p_lo + 255) / 256, (long long)ctx->num_sms * 8));
    double* partial = (double*)ws_get(ctx, WS_REDUCE, sizeof(double) * (size_t)nbk);
    if (kind == DFT_XC_PBE96)
        slab_xc_energy_kernel<1><<<nbk, 256, 0, ctx->stream>>>(s, p_lo, p_hi, na, nb, partial);
    else
        slab_xc_energy_kernel<0><<<nbk, 256, 0, ctx->stream>>>(s, p_lo, p_hi, na, nb, partial);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    double* h = pinned(ctx, (size_t)nbk);
    DFT_CUDA(cudaMemcpyAsync(h, partial, sizeof(double) * (size_t)nbk, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    double e = 0.0;
    for (int b = 0; b < nbk; ++b) e += h[b];
    return e;
}

void zslab_gram(dft_context* ctx, const Grid& g, int z_lo, int z_hi, int own_lo, int own_hi, const double* A,
                long long lda, int ka, const double* B, long long ldb, int kb, int precision, std::vector<double>& C) {
    check_slab(g, z_lo, z_hi);
    if (own_lo >= own_hi || own_lo < z_lo || own_hi > z_hi)
        fail(DFT_INVALID_ARGUMENT, "owned planes must be a non-empty range inside the slab");
    const long long slab_n = (long long)g.nx * g.ny * (z_hi - z_lo);
    if (lda < slab_n || ldb < slab_n) fail(DFT_INVALID_ARGUMENT, "lda and ldb must be >= nx*ny*(z_hi - z_lo)");
    const Grid own = slab_grid(g, own_lo, own_hi);
    const long long off = (long long)(own_lo - z_lo) * g.nx * g.ny;
    if (precision == 1) gram_tc(ctx, own, A + off, lda, ka, B + off, ldb, kb, C);
    else gram_fp64(ctx, own, A + off, lda, ka, B + off, ldb, kb, C);
}

}  // namespace dftb
