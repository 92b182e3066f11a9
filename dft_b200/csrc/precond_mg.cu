// Multigrid preconditioner for the block eigensolver: one V(2,2) cycle from zero for
// (T + sigma_a) t_a = r_a per correction band, T = -1/2 lap_h with psi = 0 outside the box
// (the kinetic operator of applyMolecularKohnShamHamiltonian, KohnShamHamiltonianMolecule.cpp:90-166),
// sigma_a = max(-theta_a, 1 Ha).  All bands advance together: every kernel takes the band
// index from blockIdx.y.  The reference preconditions with the diagonal of H - theta
// (EigenvalueSolverMolecule.cpp:521-555); this is an option of the block solver, not the
// reference's behaviour.
//
// Per level the equation is (den + c_a) t_p - sum_nb w_d t_nb = s * src_p over every grid point
// (neighbours outside the box are zero), with den = 2 (ix2 + iy2 + iz2), w_d = 1/h_d^2,
// c_a = 2 sigma_a and s = 2 on the finest level (the residual r), 1 on coarse levels.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "neural.h"
#include "ops.h"

namespace dftb {
namespace {

__device__ __forceinline__ double nb_sum_open(const Grid& g, const double* v, long long p) {
    const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
    const long long sxy = (long long)g.nx * g.ny;
    double s = 0.0;
    if (i > 0) s += g.ix2 * v[p - 1];
    if (i + 1 < g.nx) s += g.ix2 * v[p + 1];
    if (j > 0) s += g.iy2 * v[p - g.nx];
    if (j + 1 < g.ny) s += g.iy2 * v[p + g.nx];
    if (k > 0) s += g.iz2 * v[p - sxy];
    if (k + 1 < g.nz) s += g.iz2 * v[p + sxy];
    return s;
}

// Fine-level kernels march z over a column (i, j) per thread, like the H psi kernel: the z
// neighbours come from registers and no point index is divided.  blockIdx.z = band * nzc + chunk.
constexpr int PX = 32, PY = 8;

// out = v + omega ((sum + s src) / (den + c) - v); v == nullptr means v = 0
__global__ void __launch_bounds__(PX* PY) pc_smooth_kernel(Grid g, long long ld, const double* __restrict__ src,
                                                          double s, const double* __restrict__ shift,
                                                          const double* __restrict__ v, double* __restrict__ out,
                                                          double omega, int zc, int nzc) {
    const int i = blockIdx.x * PX + threadIdx.x, j = blockIdx.y * PY + threadIdx.y;
    const int a = blockIdx.z / nzc, kc = blockIdx.z - a * nzc;
    if (i >= g.nx || j >= g.ny) return;
    const double d = 2.0 * (g.ix2 + g.iy2 + g.iz2) + shift[a];
    const double* sa = src + (long long)a * ld;
    double* oa = out + (long long)a * ld;
    const long long sxy = (long long)g.nx * g.ny;
    const int kb = kc * zc, ke = min(g.nz, kb + zc);
    long long p = (long long)kb * sxy + (long long)j * g.nx + i;
    if (!v) {
        for (int k = kb; k < ke; ++k, p += sxy) oa[p] = omega * s * sa[p] / d;
        return;
    }
    const double* va = v + (long long)a * ld;
    const bool xl = i > 0, xr = i + 1 < g.nx, yl = j > 0, yr = j + 1 < g.ny;
    double below = kb > 0 ? va[p - sxy] : 0.0, cur = va[p];
    for (int k = kb; k < ke; ++k, p += sxy) {
        const double above = k + 1 < g.nz ? va[p + sxy] : 0.0;
        double sum = g.iz2 * (below + above);
        if (xl) sum += g.ix2 * va[p - 1];
        if (xr) sum += g.ix2 * va[p + 1];
        if (yl) sum += g.iy2 * va[p - g.nx];
        if (yr) sum += g.iy2 * va[p + g.nx];
        const double vj = (sum + s * sa[p]) / d;
        oa[p] = cur + omega * (vj - cur);
        below = cur;
        cur = above;
    }
}

// r = s src - ((den + c) v - sum)
__global__ void __launch_bounds__(PX* PY) pc_residual_kernel(Grid g, long long ld, const double* __restrict__ src,
                                                            double s, const double* __restrict__ shift,
                                                            const double* __restrict__ v, double* __restrict__ r,
                                                            int zc, int nzc) {
    const int i = blockIdx.x * PX + threadIdx.x, j = blockIdx.y * PY + threadIdx.y;
    const int a = blockIdx.z / nzc, kc = blockIdx.z - a * nzc;
    if (i >= g.nx || j >= g.ny) return;
    const double d = 2.0 * (g.ix2 + g.iy2 + g.iz2) + shift[a];
    const double* sa = src + (long long)a * ld;
    const double* va = v + (long long)a * ld;
    double* ra = r + (long long)a * ld;
    const long long sxy = (long long)g.nx * g.ny;
    const int kb = kc * zc, ke = min(g.nz, kb + zc);
    long long p = (long long)kb * sxy + (long long)j * g.nx + i;
    const bool xl = i > 0, xr = i + 1 < g.nx, yl = j > 0, yr = j + 1 < g.ny;
    double below = kb > 0 ? va[p - sxy] : 0.0, cur = va[p];
    for (int k = kb; k < ke; ++k, p += sxy) {
        const double above = k + 1 < g.nz ? va[p + sxy] : 0.0;
        double sum = g.iz2 * (below + above);
        if (xl) sum += g.ix2 * va[p - 1];
        if (xr) sum += g.ix2 * va[p + 1];
        if (yl) sum += g.iy2 * va[p - g.nx];
        if (yr) sum += g.iy2 * va[p + g.nx];
        ra[p] = s * sa[p] - (d * cur - sum);
        below = cur;
        cur = above;
    }
}

// launch shape of the column kernels for nb fields: z chunks long enough to amortise the march,
// enough blocks to fill the machine; gridDim.z = nb * nzc must stay below 65536
struct ColShape {
    dim3 grid, block;
    int zc, nzc;
};
ColShape col_shape(dft_context* ctx, const Grid& g, int nb) {
    const int bx = (g.nx + PX - 1) / PX, by = (g.ny + PY - 1) / PY;
    int zc = 32;
    while (zc > 4 && (long long)bx * by * nb * ((g.nz + zc - 1) / zc) < 4LL * ctx->num_sms) zc >>= 1;
    int nzc = (g.nz + zc - 1) / zc;
    while ((long long)nb * nzc > 65535) {
        zc *= 2;
        nzc = (g.nz + zc - 1) / zc;
    }
    return {dim3(bx, by, nb * nzc), dim3(PX, PY), zc, nzc};
}

// Restriction along one axis (transposed trilinear weights times h/H), per band.
__global__ void pc_restrict_axis_kernel(const double* __restrict__ in, long long in_ld, double* __restrict__ out,
                                        long long out_ld, int n0, int n1, int n2, int ax, int nc, double h,
                                        double H) {
    const int a = blockIdx.y;
    in += (long long)a * in_ld;
    out += (long long)a * out_ld;
    int od[3] = {n0, n1, n2};
    const int nf = od[ax];
    od[ax] = nc;
    const long long nout = (long long)od[0] * od[1] * od[2];
    const long long s_in[3] = {1, n0, (long long)n0 * n1};
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nout; q += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        idx[0] = (int)(q % od[0]);
        idx[1] = (int)((q / od[0]) % od[1]);
        idx[2] = (int)(q / ((long long)od[0] * od[1]));
        const int I = idx[ax];
        const double X = I * H;
        const int flo = max(0, (int)ceil((X - H) / h));
        const int fhi = min(nf - 1, (int)floor((X + H) / h));
        long long b = 0;
        for (int d = 0; d < 3; ++d)
            if (d != ax) b += idx[d] * s_in[d];
        double acc = 0.0;
        for (int fi = flo; fi <= fhi; ++fi) {
            const double wgt = 1.0 - fabs(fi * h - X) / H;
            if (wgt > 0.0) acc += wgt * in[b + fi * s_in[ax]];
        }
        out[q] = acc * (h / H);
    }
}

// v += trilinear interpolation of the coarse correction e, at every fine point.  One thread per
// fine (i, j) column: the x/y cells and weights are found once, z steps along the column.
__global__ void __launch_bounds__(256) pc_prolong_add_kernel(Grid f, long long fld, Grid c, long long cld,
                                                             const double* __restrict__ e, double* __restrict__ v,
                                                             int zc, int nzc) {
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
    const int a = blockIdx.z / nzc, kc = blockIdx.z - a * nzc;
    if (i >= f.nx || j >= f.ny) return;
    e += (long long)a * cld;
    v += (long long)a * fld;
    const double ux = i * f.dx / c.dx, uy = j * f.dy / c.dy;
    const int Ix = min(max((int)floor(ux), 0), c.nx - 2), Iy = min(max((int)floor(uy), 0), c.ny - 2);
    const double wx = fmin(fmax(ux - Ix, 0.0), 1.0), wy = fmin(fmax(uy - Iy, 0.0), 1.0);
    const long long cxy = (long long)c.nx * c.ny;
    const long long b00 = (long long)Iy * c.nx + Ix;
    const long long fxy = (long long)f.nx * f.ny;
    const int kb = kc * zc, ke = min(f.nz, kb + zc);
    for (int k = kb; k < ke; ++k) {
        const double uz = k * f.dz / c.dz;
        const int Iz = min(max((int)floor(uz), 0), c.nz - 2);
        const double wz = fmin(fmax(uz - Iz, 0.0), 1.0);
        const double* e0 = e + (long long)Iz * cxy + b00;
        const double* e1 = e0 + cxy;
        const double p0 = (1.0 - wy) * ((1.0 - wx) * e0[0] + wx * e0[1]) + wy * ((1.0 - wx) * e0[c.nx] + wx * e0[c.nx + 1]);
        const double p1 = (1.0 - wy) * ((1.0 - wx) * e1[0] + wx * e1[1]) + wy * ((1.0 - wx) * e1[c.nx] + wx * e1[c.nx + 1]);
        v[(long long)k * fxy + (long long)j * f.nx + i] += (1.0 - wz) * p0 + wz * p1;
    }
}

// Coarsest level: `sweeps` Jacobi sweeps from zero, one block per band, in shared memory.
constexpr int PC_COARSEST_MAX = 12288;
__global__ void __launch_bounds__(1024) pc_coarsest_kernel(Grid g, long long ld, const double* __restrict__ src,
                                                           double s, const double* __restrict__ shift,
                                                           double* __restrict__ e, int sweeps) {
    extern __shared__ double sm[];
    const int a = blockIdx.x;
    const int n = (int)g.N;
    src += (long long)a * ld;
    e += (long long)a * ld;
    double* x = sm;
    double* y = sm + n;
    for (int p = threadIdx.x; p < n; p += blockDim.x) x[p] = 0.0;
    __syncthreads();
    const double d = 2.0 * (g.ix2 + g.iy2 + g.iz2) + shift[a];
    for (int it = 0; it < sweeps; ++it) {
        const double* cur = (it & 1) ? y : x;
        double* nxt = (it & 1) ? x : y;
        for (int p = threadIdx.x; p < n; p += blockDim.x) nxt[p] = (nb_sum_open(g, cur, p) + s * src[p]) / d;
        __syncthreads();
    }
    const double* res = (sweeps & 1) ? y : x;
    for (int p = threadIdx.x; p < n; p += blockDim.x) e[p] = res[p];
}

// shift[a] = c for every field (the screened Poisson equation of the Kerker mixer)
__global__ void pc_fill_kernel(int nb, double c, double* __restrict__ shift) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nb; a += gridDim.x * blockDim.x) shift[a] = c;
}

// c_a = 2 max(-theta[src[a]], 1 Ha): the shift of each correction band, from the Ritz values
__global__ void pc_shift_kernel(int nb, const double* __restrict__ theta, const int* __restrict__ src,
                                double* __restrict__ shift) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nb; a += gridDim.x * blockDim.x)
        shift[a] = 2.0 * fmax(-theta[src[a]], 1.0);
}

__global__ void pc_gather_kernel(long long n, long long ld, const double* __restrict__ R, const int* __restrict__ srcmap,
                                 double* __restrict__ out) {
    const int a = blockIdx.y;
    const double* r = R + (long long)(srcmap ? srcmap[a] : a) * ld;
    double* o = out + (long long)a * ld;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        o[p] = r[p];
}

struct PCLevel {
    Grid g;
    long long ld;
    double *src, *v, *tmp, *res, *t1, *t2;
};

Grid pc_coarse(const Grid& g) {
    dft_grid d{coarse_points(g.nx), coarse_points(g.ny), coarse_points(g.nz), g.xmin, g.xmax, g.ymin,
               g.ymax,          g.zmin,          g.zmax};
    return make_grid(&d);
}

inline dim3 pc_grid(dft_context* ctx, long long n, int nb) {
    long long bx = (n + 255) / 256;
    const long long cap = std::max<long long>(1, (long long)ctx->num_sms * 8 / std::max(nb, 1));
    bx = std::max<long long>(1, std::min(bx, std::max<long long>(cap, 4)));
    return dim3((unsigned)bx, (unsigned)nb);
}

void pc_smooth(dft_context* ctx, PCLevel& l, double s, const double* shift, int nb, int n, bool from_zero) {
    const ColShape c = col_shape(ctx, l.g, nb);
    for (int k = 0; k < n; ++k) {
        const double* v = (from_zero && k == 0) ? nullptr : l.v;
        pc_smooth_kernel<<<c.grid, c.block, 0, ctx->stream>>>(l.g, l.ld, l.src, s, shift, v, l.tmp, 0.8, c.zc, c.nzc);
        std::swap(l.v, l.tmp);
    }
    count_launch(ctx, n);
}

void pc_vcycle(dft_context* ctx, std::vector<PCLevel>& L, size_t i, double s, const double* shift, int nb) {
    PCLevel& l = L[i];
    if (i + 1 == L.size()) {
        pc_coarsest_kernel<<<nb, 1024, sizeof(double) * 2 * (size_t)l.g.N, ctx->stream>>>(
            l.g, l.ld, l.src, s, shift, l.v, 8 * std::max({l.g.nx, l.g.ny, l.g.nz}));
        count_launch(ctx);
        return;
    }
    pc_smooth(ctx, l, s, shift, nb, 2, true);
    {
        const ColShape c = col_shape(ctx, l.g, nb);
        pc_residual_kernel<<<c.grid, c.block, 0, ctx->stream>>>(l.g, l.ld, l.src, s, shift, l.v, l.res, c.zc, c.nzc);
    }
    PCLevel& c = L[i + 1];
    const Grid& f = l.g;
    pc_restrict_axis_kernel<<<pc_grid(ctx, (long long)f.nz * f.ny * c.g.nx, nb), 256, 0, ctx->stream>>>(
        l.res, l.ld, l.t1, (long long)f.nz * f.ny * c.g.nx, f.nx, f.ny, f.nz, 0, c.g.nx, f.dx, c.g.dx);
    pc_restrict_axis_kernel<<<pc_grid(ctx, (long long)f.nz * c.g.ny * c.g.nx, nb), 256, 0, ctx->stream>>>(
        l.t1, (long long)f.nz * f.ny * c.g.nx, l.t2, (long long)f.nz * c.g.ny * c.g.nx, c.g.nx, f.ny, f.nz, 1, c.g.ny,
        f.dy, c.g.dy);
    pc_restrict_axis_kernel<<<pc_grid(ctx, c.g.N, nb), 256, 0, ctx->stream>>>(
        l.t2, (long long)f.nz * c.g.ny * c.g.nx, c.src, c.ld, c.g.nx, c.g.ny, f.nz, 2, c.g.nz, f.dz, c.g.dz);
    count_launch(ctx, 4);
    pc_vcycle(ctx, L, i + 1, 1.0, shift, nb);
    {
        const ColShape cs = col_shape(ctx, f, nb);
        pc_prolong_add_kernel<<<cs.grid, cs.block, 0, ctx->stream>>>(f, l.ld, c.g, c.ld, c.v, l.v, cs.zc, cs.nzc);
    }
    count_launch(ctx);
    pc_smooth(ctx, l, s, shift, nb, 2, false);
    DFT_LAUNCH_CHECK();
}

// One V(2,2) cycle from zero, all nb fields together, for (den + shift_a) t - sum_nb w t_nb =
// s * R_{src[a]} on g (src_dev == nullptr: field a itself), into T.  shift_dev must not live in
// the WS_PG2 workspace.
void vcycle_batch(dft_context* ctx, const Grid& g, const double* R, const int* src_dev, int nb, const double* shift,
                  double s, double* T, long long ld) {
    std::vector<PCLevel> L;
    PCLevel f{};
    f.g = g;
    f.ld = ld;
    L.push_back(f);
    Grid cur = g;
    while (cur.N > PC_COARSEST_MAX || std::min({cur.nx, cur.ny, cur.nz}) > 9) {
        const Grid c = pc_coarse(cur);
        if (c.nx == cur.nx && c.ny == cur.ny && c.nz == cur.nz) break;
        PCLevel l{};
        l.g = c;
        l.ld = c.N;
        L.push_back(l);
        cur = c;
        if (L.size() >= 10) break;
    }
    if (L.back().g.N > PC_COARSEST_MAX) fail(DFT_INVALID_ARGUMENT, "grid too small or anisotropic for multigrid");
    // slab: per band, fine tmp/res and src copy; coarse levels src/v/tmp/res; restriction temps
    size_t per_band = 3 * (size_t)ld + 16;
    for (size_t i = 0; i < L.size(); ++i) {
        if (i > 0) per_band += 4 * (size_t)L[i].g.N + 8;
        if (i + 1 < L.size()) {
            const Grid& a = L[i].g;
            const Grid& c = L[i + 1].g;
            per_band += (size_t)a.nz * a.ny * c.nx + (size_t)a.nz * c.ny * c.nx + 8;
        }
    }
    double* slab = (double*)ws_get(ctx, WS_PG2, sizeof(double) * (per_band * nb + 64));
    double* p = slab;
    auto take = [&](size_t n) {
        double* q = p;
        p += (n * nb + 1) / 2 * 2;
        return q;
    };
    L[0].src = take((size_t)ld);
    L[0].tmp = take((size_t)ld);
    L[0].res = take((size_t)ld);
    L[0].v = T;
    for (size_t i = 0; i < L.size(); ++i) {
        if (i > 0) {
            L[i].src = take((size_t)L[i].g.N);
            L[i].v = take((size_t)L[i].g.N);
            L[i].tmp = take((size_t)L[i].g.N);
            L[i].res = take((size_t)L[i].g.N);
        }
        if (i + 1 < L.size()) {
            const Grid& a = L[i].g;
            const Grid& c = L[i + 1].g;
            L[i].t1 = take((size_t)a.nz * a.ny * c.nx);
            L[i].t2 = take((size_t)a.nz * c.ny * c.nx);
        }
    }
    static bool attr = false;
    if (!attr) {
        DFT_CUDA(cudaFuncSetAttribute(pc_coarsest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double) * 2 * PC_COARSEST_MAX)));
        attr = true;
    }
    pc_gather_kernel<<<pc_grid(ctx, g.N, nb), 256, 0, ctx->stream>>>(g.N, ld, R, src_dev, L[0].src);
    count_launch(ctx);
    pc_vcycle(ctx, L, 0, s, shift, nb);
    if (L[0].v != T)
        DFT_CUDA(cudaMemcpy2DAsync(T, sizeof(double) * ld, L[0].v, sizeof(double) * ld, sizeof(double) * g.N, nb,
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    DFT_LAUNCH_CHECK();
}

}  // namespace

void precondition_multigrid(dft_context* ctx, const Grid& g, const double* R, const int* src_dev, int nb,
                            const double* theta_dev, double* T, long long ld) {
    if (nb <= 0) return;
    // shifts c_a = 2 sigma_a, computed on the device (no host round trip)
    double* shift = (double*)ws_get(ctx, WS_PG3, sizeof(double) * (size_t)nb + 64);
    pc_shift_kernel<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(nb, theta_dev, src_dev, shift);
    count_launch(ctx);
    vcycle_batch(ctx, g, R, src_dev, nb, shift, 2.0, T, ld);
}

namespace {
__global__ void pc_sigma_shift_kernel(int nb, const double* __restrict__ sigma, double* __restrict__ shift) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < nb; a += gridDim.x * blockDim.x) shift[a] = 2.0 * sigma[a];
}
__global__ void pc_add_kernel(long long n, long long ld, const double* __restrict__ e, double* __restrict__ x) {
    const int a = blockIdx.y;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        x[(long long)a * ld + p] += e[(long long)a * ld + p];
}
}  // namespace

void helmholtz_refine(dft_context* ctx, const Grid& g, const double* R, int nb, const double* sigma_dev, double* X,
                      long long ld, int cycles, double* res, double* e) {
    if (nb <= 0) return;
    double* shift = (double*)ws_get(ctx, WS_PG3, sizeof(double) * (size_t)nb + 64);
    pc_sigma_shift_kernel<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(nb, sigma_dev, shift);
    count_launch(ctx);
    vcycle_batch(ctx, g, R, nullptr, nb, shift, 2.0, X, ld);
    for (int c = 1; c < cycles; ++c) {
        // res = 2 R - ((den + 2 sigma) X - sum), the equation's residual in the cycle's scaling
        const ColShape cs = col_shape(ctx, g, nb);
        pc_residual_kernel<<<cs.grid, cs.block, 0, ctx->stream>>>(g, ld, R, 2.0, shift, X, res, cs.zc, cs.nzc);
        count_launch(ctx);
        vcycle_batch(ctx, g, res, nullptr, nb, shift, 1.0, e, ld);
        pc_add_kernel<<<pc_grid(ctx, g.N, nb), 256, 0, ctx->stream>>>(g.N, ld, e, X);
        count_launch(ctx);
        DFT_LAUNCH_CHECK();
    }
}

void screened_poisson_vcycle(dft_context* ctx, const Grid& g, const double* src, int nb, double q2, double* x,
                             long long ld, int cycles) {
    if (nb <= 0) return;
    if (!(q2 > 0.0) || !std::isfinite(q2)) fail(DFT_INVALID_ARGUMENT, "screening q^2 must be > 0");
    if (cycles < 1) fail(DFT_INVALID_ARGUMENT, "cycles must be >= 1");
    double* shift = (double*)ws_get(ctx, WS_PG3, sizeof(double) * (size_t)nb + 64);
    pc_fill_kernel<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(nb, q2, shift);
    count_launch(ctx);
    vcycle_batch(ctx, g, src, nullptr, nb, shift, 1.0, x, ld);
    if (cycles == 1) return;
    // iterative refinement: res = src - (-lap + q2) x, e = V-cycle(res), x += e
    double* scratch = (double*)ws_get(ctx, WS_PG4, sizeof(double) * 2 * (size_t)nb * ld);
    double *res = scratch, *e = scratch + (size_t)nb * ld;
    for (int c = 1; c < cycles; ++c) {
        const ColShape cs = col_shape(ctx, g, nb);
        pc_residual_kernel<<<cs.grid, cs.block, 0, ctx->stream>>>(g, ld, src, 1.0, shift, x, res, cs.zc, cs.nzc);
        count_launch(ctx);
        vcycle_batch(ctx, g, res, nullptr, nb, shift, 1.0, e, ld);
        pc_add_kernel<<<pc_grid(ctx, g.N, nb), 256, 0, ctx->stream>>>(g.N, ld, e, x);
        count_launch(ctx);
        DFT_LAUNCH_CHECK();
    }
}

}  // namespace dftb
