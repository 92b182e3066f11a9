// Start values for the Jacobi Poisson solve (no counterpart in the reference, whose solve
// always starts from zero, HartreePotentialMolecule.cpp:152-155): nested coarse grids, an
// optional network correction (neural.cu) and multigrid V-cycles.  The Jacobi solve that
// follows keeps the reference's stop rule, so every start ends at a Jacobi fixed point to
// the same tolerance; only the number of fine-grid sweeps changes.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "common.cuh"
#include "neural.h"
#include "ops.h"

namespace dftb {

int coarse_points(int n) { return std::max(5, (int)std::lround((n - 1) / 2.0) + 1); }

namespace {

// ---------------------------------------------------------------- coarse grid ----------
// Restriction along one axis with the transposed trilinear (hat) weights times h/H, so the
// total charge sum rho dV is kept.  in: (n0, n1, n2) with axis `ax` of length nf; out: the
// same with that axis of length nc.  x_f = lo + f h, X_I = lo + I H.
__global__ void restrict_axis_kernel(const double* __restrict__ in, double* __restrict__ out, int n0, int n1, int n2,
                                     int ax, int nc, double h, double H) {
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
        double s = 0.0;
        for (int fi = flo; fi <= fhi; ++fi) {
            const double wgt = 1.0 - fabs(fi * h - X) / H;
            if (wgt > 0.0) s += wgt * in[b + fi * s_in[ax]];
        }
        out[q] = s * (h / H);
    }
}

// Trilinear interpolation of the coarse solution (same bounds) onto the fine interior.
__global__ void prolong_kernel(Grid f, Grid c, const double* __restrict__ vc, double* __restrict__ out) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < f.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % f.nx), j = (int)((p / f.nx) % f.ny), k = (int)(p / ((long long)f.nx * f.ny));
        const bool face = i == 0 || i + 1 == f.nx || j == 0 || j + 1 == f.ny || k == 0 || k + 1 == f.nz;
        if (face) {
            out[p] = 0.0;
            continue;
        }
        const double u[3] = {i * f.dx / c.dx, j * f.dy / c.dy, k * f.dz / c.dz};
        const int m[3] = {c.nx, c.ny, c.nz};
        int I[3];
        double w[3];
        for (int d = 0; d < 3; ++d) {
            I[d] = min(max((int)floor(u[d]), 0), m[d] - 2);
            w[d] = fmin(fmax(u[d] - I[d], 0.0), 1.0);
        }
        double s = 0.0;
        for (int t = 0; t < 8; ++t) {
            const int a = t & 1, b = (t >> 1) & 1, cc = t >> 2;
            const double wt = (a ? w[0] : 1.0 - w[0]) * (b ? w[1] : 1.0 - w[1]) * (cc ? w[2] : 1.0 - w[2]);
            s += wt * vc[((long long)(I[2] + cc) * c.ny + (I[1] + b)) * c.nx + (I[0] + a)];
        }
        out[p] = s;
    }
}

// s = max |v| (1 if zero): the network's input/output scale, kept on the device.
__global__ void absmax_kernel(long long n, const double* __restrict__ v, double* __restrict__ s) {
    __shared__ double sh[32];
    double m = 0.0;
    for (long long p = threadIdx.x; p < n; p += blockDim.x) m = fmax(m, fabs(v[p]));
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sh[w]);
        *s = r > 0.0 ? r : 1.0;
    }
}

__global__ void sum_kernel(long long n, const double* __restrict__ v, double* __restrict__ out) {
    __shared__ double sh[32];
    double m = 0.0;
    for (long long p = threadIdx.x; p < n; p += blockDim.x) m += v[p];
    m = warp_sum(m);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sh[w];
        *out = r;
    }
}

struct Gauss {
    double x, y, z, a, inv2w2;
};
__global__ void gauss_density_kernel(Grid g, const Gauss* __restrict__ gs, int k, double* __restrict__ rho) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), kk = (int)(p / ((long long)g.nx * g.ny));
        const double x = g.xmin + i * g.dx, y = g.ymin + j * g.dy, z = g.zmin + kk * g.dz;
        double s = 0.0;
        for (int q = 0; q < k; ++q) {
            const double dx = x - gs[q].x, dy = y - gs[q].y, dz = z - gs[q].z;
            s += gs[q].a * exp(-(dx * dx + dy * dy + dz * dz) * gs[q].inv2w2);
        }
        rho[p] = s;
    }
}

__global__ void scale_kernel(long long n, double* __restrict__ v, double c) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        v[p] *= c;
}

inline int blocks_for(dft_context* ctx, long long n, int per = 256) {
    const long long b = (n + per - 1) / per;
    return (int)std::max<long long>(1, std::min<long long>(b, (long long)ctx->num_sms * 8));
}

Grid coarse_grid(const Grid& g) {
    dft_grid d{coarse_points(g.nx), coarse_points(g.ny), coarse_points(g.nz), g.xmin, g.xmax, g.ymin,
               g.ymax,          g.zmin,          g.zmax};
    return make_grid(&d);
}

// Nested coarse levels: level 0 = coarse_grid(g), level l+1 = coarse_grid(level l), while
// every axis keeps at least 17 points.  Each level is solved by multigrid cycles from the next
// coarser level's interpolated solution (full multigrid); the finest coarse level's
// solution, interpolated to g, is the start.  Faces are held at zero on every level.  All
// level arrays are carved from one slab of doubles.
struct Level {
    Grid g;
    double *t1, *t2, *rc, *vc, *vs;
};

std::vector<Level> plan_levels(const Grid& fine) {
    std::vector<Level> L;
    Grid cur = fine;
    do {
        Level l{};
        l.g = coarse_grid(cur);
        L.push_back(l);
        cur = l.g;
    } while (std::min({cur.nx, cur.ny, cur.nz}) >= 17 && L.size() < 8);
    return L;
}

size_t slab_doubles(const Grid& fine, const std::vector<Level>& L) {
    size_t n = 8;  // the scale s
    Grid prev = fine;
    for (const Level& l : L) {
        n += (size_t)prev.nz * prev.ny * l.g.nx + (size_t)prev.nz * l.g.ny * l.g.nx + 3 * (size_t)l.g.N + 8;
        prev = l.g;
    }
    return n;
}

// Carves the level arrays; returns the scale slot.
double* carve(double* slab, const Grid& fine, std::vector<Level>& L) {
    double* s = slab;
    double* p = slab + 8;
    Grid prev = fine;
    auto take = [&](size_t n) {
        double* q = p;
        p += (n + 1) / 2 * 2;  // keep 16-byte alignment
        return q;
    };
    for (Level& l : L) {
        l.t1 = take((size_t)prev.nz * prev.ny * l.g.nx);
        l.t2 = take((size_t)prev.nz * l.g.ny * l.g.nx);
        l.rc = take((size_t)l.g.N);
        l.vc = take((size_t)l.g.N);
        l.vs = take((size_t)l.g.N);
        prev = l.g;
    }
    return s;
}

// The same restriction in one pass (small fine grids, where the three passes are three
// launch latencies): out(I,J,K) = prod_d (h_d/H_d) sum_k w_z sum_j w_y sum_i w_x in(i,j,k).
// hat weights of one axis: w[t] for fine index lo + t (at most RW of them; coarse spacing
// <= 2.5 fine spacings, which coarse_points guarantees)
constexpr int RW = 6;
__device__ __forceinline__ int hat_weights(int I, double h, double H, int nf, double* w) {
    const double X = I * H;
    const int lo = max(0, (int)ceil((X - H) / h)), hi = min(nf - 1, (int)floor((X + H) / h));
#pragma unroll
    for (int t = 0; t < RW; ++t) {
        const int i = lo + t;
        const double v = i <= hi ? 1.0 - fabs(i * h - X) / H : 0.0;
        w[t] = v > 0.0 ? v : 0.0;
    }
    return lo;
}

__global__ void restrict3d_kernel(const double* __restrict__ in, double* __restrict__ out, Grid f, Grid c) {
    const double scale = (f.dx / c.dx) * (f.dy / c.dy) * (f.dz / c.dz);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < c.N; q += (long long)gridDim.x * blockDim.x) {
        const int I = (int)(q % c.nx), J = (int)((q / c.nx) % c.ny), K = (int)(q / ((long long)c.nx * c.ny));
        double wx[RW], wy[RW], wz[RW];
        const int i0 = hat_weights(I, f.dx, c.dx, f.nx, wx);
        const int j0 = hat_weights(J, f.dy, c.dy, f.ny, wy);
        const int k0 = hat_weights(K, f.dz, c.dz, f.nz, wz);
        double sz = 0.0;
#pragma unroll
        for (int tk = 0; tk < RW; ++tk) {
            if (wz[tk] == 0.0) continue;
            double sy = 0.0;
#pragma unroll
            for (int tj = 0; tj < RW; ++tj) {
                if (wy[tj] == 0.0) continue;
                const double* row = in + ((long long)(k0 + tk) * f.ny + (j0 + tj)) * f.nx + i0;
                double sx = 0.0;
#pragma unroll
                for (int ti = 0; ti < RW; ++ti)
                    if (wx[ti] != 0.0) sx += wx[ti] * row[ti];
                sy += wy[tj] * sx;
            }
            sz += wz[tk] * sy;
        }
        out[q] = sz * scale;
    }
}

void restrict3(dft_context* ctx, const Grid& f, const Grid& c, const double* in, double* t1, double* t2,
               double* out) {
    if (ctx->mg_fused_restrict && f.N <= 64LL * 64 * 64 && c.dx <= 2.5 * f.dx && c.dy <= 2.5 * f.dy &&
        c.dz <= 2.5 * f.dz) {
        restrict3d_kernel<<<blocks_for(ctx, c.N), 256, 0, ctx->stream>>>(in, out, f, c);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        return;
    }
    restrict_axis_kernel<<<blocks_for(ctx, (long long)f.nz * f.ny * c.nx), 256, 0, ctx->stream>>>(
        in, t1, f.nx, f.ny, f.nz, 0, c.nx, f.dx, c.dx);
    restrict_axis_kernel<<<blocks_for(ctx, (long long)f.nz * c.ny * c.nx), 256, 0, ctx->stream>>>(
        t1, t2, c.nx, f.ny, f.nz, 1, c.ny, f.dy, c.dy);
    restrict_axis_kernel<<<blocks_for(ctx, c.N), 256, 0, ctx->stream>>>(t2, out, c.nx, c.ny, f.nz, 2, c.nz, f.dz,
                                                                       c.dz);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 3);
}

// vup = the nested coarse solution interpolated to g; *s (device) = max |level-0 solution|.
// Returns the Jacobi sweeps of all coarse levels.
long coarse_solve(dft_context* ctx, double* slab, const Grid& g, const double* rho, double* vup, double** s_out,
                  Grid* gc_out) {
    std::vector<Level> L = plan_levels(g);
    double* s = carve(slab, g, L);
    const bool zero = faces_exact(g);  // the coarse boundary follows the fine grid's
    const double* src = rho;
    Grid sg = g;
    for (Level& l : L) {
        restrict3(ctx, sg, l.g, src, l.t1, l.t2, l.rc);
        src = l.rc;
        sg = l.g;
    }
    long cycles = 0;
    (void)zero;
    for (int i = (int)L.size() - 1; i >= 0; --i) {
        Level& l = L[i];
        // each level from the next coarser level's interpolated solution (zero on the coarsest)
        if (i + 1 < (int)L.size())
            DFT_CUDA(cudaMemcpyAsync(l.vc, l.vs, sizeof(double) * (size_t)l.g.N, cudaMemcpyDeviceToDevice, ctx->stream));
        else
            DFT_CUDA(cudaMemsetAsync(l.vc, 0, sizeof(double) * (size_t)l.g.N, ctx->stream));
        cycles += multigrid(ctx, l.g, l.rc, l.vc, 1e-7, 20, nullptr);
        const Grid& to = i == 0 ? g : L[i - 1].g;
        double* dst = i == 0 ? vup : L[i - 1].vs;
        prolong_kernel<<<blocks_for(ctx, to.N), 256, 0, ctx->stream>>>(to, l.g, l.vc, dst);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
    absmax_kernel<<<1, 1024, 0, ctx->stream>>>(L[0].g.N, L[0].vc, s);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    if (s_out) *s_out = s;
    if (gc_out) *gc_out = L[0].g;
    return cycles;
}

double* coarse_slab(dft_context* ctx, const Grid& g) {
    const std::vector<Level> L = plan_levels(g);
    return (double*)ws_get(ctx, WS_PG0, sizeof(double) * slab_doubles(g, L));
}

// ---------------------------------------------------------------- multigrid ------------
// Discrete equation per level (faces fixed): den v_p - sum_nb w_d v_nb = src_p, with
// den = 2 (ix2 + iy2 + iz2) and w_d = 1/h_d^2; the fine level's source is 4 pi rho.
__device__ __forceinline__ double nb_sum(const Grid& g, const double* v, long long p) {
    const long long sxy = (long long)g.nx * g.ny;
    return g.ix2 * (v[p - 1] + v[p + 1]) + g.iy2 * (v[p - g.nx] + v[p + g.nx]) + g.iz2 * (v[p - sxy] + v[p + sxy]);
}
__device__ __forceinline__ bool on_face(const Grid& g, long long p) {
    const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
    return i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz;
}

// weighted Jacobi: out = v + omega ((sum + s*src)/den - v); faces copied
__global__ void mg_smooth_kernel(Grid g, const double* __restrict__ src, double sscale, const double* __restrict__ v,
                                 double* __restrict__ out, double omega) {
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        if (on_face(g, p)) {
            out[p] = v[p];
            continue;
        }
        const double vj = (nb_sum(g, v, p) + sscale * src[p]) / den;
        out[p] = v[p] + omega * (vj - v[p]);
    }
}

// r = s*src - (den v - sum) on the interior, 0 on faces; folds max |r| into *rmax (as the
// bits of a non-negative double) when rmax is not null
__global__ void mg_residual_kernel(Grid g, const double* __restrict__ src, double sscale, const double* __restrict__ v,
                                   double* __restrict__ r, unsigned long long* __restrict__ rmax) {
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    double m = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        double rr = 0.0;
        if (!on_face(g, p)) rr = sscale * src[p] - (den * v[p] - nb_sum(g, v, p));
        r[p] = rr;
        m = fmax(m, fabs(rr));
    }
    if (rmax) {
        m = warp_max(m);
        if ((threadIdx.x & 31) == 0) atomicMax(rmax, (unsigned long long)__double_as_longlong(m));
    }
}

// v += trilinear interpolation of the coarse correction e (interior of the fine grid)
__global__ void prolong_add_kernel(Grid f, Grid c, const double* __restrict__ e, double* __restrict__ v) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < f.N; p += (long long)gridDim.x * blockDim.x) {
        if (on_face(f, p)) continue;
        const int i = (int)(p % f.nx), j = (int)((p / f.nx) % f.ny), k = (int)(p / ((long long)f.nx * f.ny));
        const double u[3] = {i * f.dx / c.dx, j * f.dy / c.dy, k * f.dz / c.dz};
        const int m[3] = {c.nx, c.ny, c.nz};
        int I[3];
        double w[3];
        for (int d = 0; d < 3; ++d) {
            I[d] = min(max((int)floor(u[d]), 0), m[d] - 2);
            w[d] = fmin(fmax(u[d] - I[d], 0.0), 1.0);
        }
        double s = 0.0;
        for (int t = 0; t < 8; ++t) {
            const int a = t & 1, b = (t >> 1) & 1, cc = t >> 2;
            const double wt = (a ? w[0] : 1.0 - w[0]) * (b ? w[1] : 1.0 - w[1]) * (cc ? w[2] : 1.0 - w[2]);
            s += wt * e[((long long)(I[2] + cc) * c.ny + (I[1] + b)) * c.nx + (I[0] + a)];
        }
        v[p] += s;
    }
}

// Coarsest level: `sweeps` red-black SOR sweeps (relaxation omega) from zero in one block's
// shared memory.  With the optimal omega the error falls by omega - 1 per sweep instead of the
// Jacobi spectral radius, so a few sweeps do what 8 Jacobi sweeps per point of the longest axis did.
constexpr int MG_COARSEST_MAX = 12288;
__global__ void __launch_bounds__(1024) mg_coarsest_kernel(Grid g, const double* __restrict__ src,
                                                           double* __restrict__ e, int sweeps, double omega) {
    extern __shared__ double sm[];
    const int n = (int)g.N;
    double* a = sm;
    for (int p = threadIdx.x; p < n; p += blockDim.x) a[p] = 0.0;
    __syncthreads();
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    // omega == 1: plain Jacobi sweeps (the sweep reads the previous iterate: a second array)
    if (omega == 1.0) {
        double* b = sm + n;
        for (int p = threadIdx.x; p < n; p += blockDim.x) b[p] = 0.0;
        __syncthreads();
        for (int s = 0; s < sweeps; ++s) {
            const double* cur = (s & 1) ? b : a;
            double* nxt = (s & 1) ? a : b;
            for (int p = threadIdx.x; p < n; p += blockDim.x)
                if (!on_face(g, p)) nxt[p] = (nb_sum(g, cur, p) + src[p]) / den;
            __syncthreads();
        }
        if (sweeps & 1)
            for (int p = threadIdx.x; p < n; p += blockDim.x) a[p] = b[p];
        __syncthreads();
    } else {
        for (int s = 0; s < sweeps; ++s)
            for (int colour = 0; colour < 2; ++colour) {
                for (int p = threadIdx.x; p < n; p += blockDim.x) {
                    const int i = p % g.nx, j = (p / g.nx) % g.ny, k = p / (g.nx * g.ny);
                    if (((i + j + k) & 1) != colour || on_face(g, p)) continue;
                    const double gs = (nb_sum(g, a, p) + src[p]) / den;
                    a[p] += omega * (gs - a[p]);
                }
                __syncthreads();
            }
    }
    for (int p = threadIdx.x; p < n; p += blockDim.x) e[p] = a[p];
}

// Optimal SOR relaxation for the 7-point operator on grid g (from the Jacobi spectral radius
// of the Dirichlet problem) and the sweeps that cut the error by 1e-4.
void coarsest_sor(const Grid& g, double* omega, int* sweeps) {
    const double pi = 3.14159265358979323846;
    const double rj = (g.ix2 * std::cos(pi / (g.nx - 1)) + g.iy2 * std::cos(pi / (g.ny - 1)) +
                       g.iz2 * std::cos(pi / (g.nz - 1))) /
                      (g.ix2 + g.iy2 + g.iz2);
    *omega = 2.0 / (1.0 + std::sqrt(std::max(0.0, 1.0 - rj * rj)));
    const double rate = std::max(*omega - 1.0, 1e-3);
    const int need = (int)std::ceil(std::log(1e-4) / std::log(rate));
    *sweeps = std::min(8 * std::max({g.nx, g.ny, g.nz}), std::max(4, need));
}

inline int mg_blocks(dft_context* ctx, long long n) {
    const long long b = (n + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(b, (long long)ctx->num_sms * 8));
}


// ---------------------------------------------------------------- multigrid solve ------
// V(2,2) cycles with weighted Jacobi (omega = 0.8) on the nested coarse grids, the same
// charge-conserving restriction and trilinear interpolation, and a coarsest-level red-black
// SOR solve in one block's shared memory.  Faces of every level are held at zero (the boundary of every grid
// whose last nodes land on the bounds).
struct MGLevel {
    Grid g;
    double *src, *v, *tmp, *res, *t1, *t2;  // t1/t2: restriction temporaries towards the next level
};

std::vector<MGLevel> mg_plan(const Grid& fine) {
    std::vector<MGLevel> L;
    MGLevel f{};
    f.g = fine;
    L.push_back(f);
    Grid cur = fine;
    while (cur.N > MG_COARSEST_MAX || std::min({cur.nx, cur.ny, cur.nz}) > 9) {
        const Grid c = coarse_grid(cur);
        if (c.nx == cur.nx && c.ny == cur.ny && c.nz == cur.nz) break;
        MGLevel l{};
        l.g = c;
        L.push_back(l);
        cur = c;
        if (L.size() >= 10) break;
    }
    return L;
}

size_t mg_doubles(const std::vector<MGLevel>& L) {
    size_t n = 16;
    for (size_t i = 0; i < L.size(); ++i) {
        const Grid& g = L[i].g;
        n += 4 * ((size_t)g.N + 2);
        if (i + 1 < L.size()) {
            const Grid& c = L[i + 1].g;
            n += (size_t)g.nz * g.ny * c.nx + (size_t)g.nz * c.ny * c.nx + 4;
        }
    }
    return n;
}

void mg_carve(double* slab, std::vector<MGLevel>& L) {
    double* p = slab + 16;
    auto take = [&](size_t n) {
        double* q = p;
        p += (n + 1) / 2 * 2;
        return q;
    };
    for (size_t i = 0; i < L.size(); ++i) {
        const Grid& g = L[i].g;
        L[i].src = i == 0 ? nullptr : take((size_t)g.N);
        L[i].v = i == 0 ? nullptr : take((size_t)g.N);
        L[i].tmp = take((size_t)g.N);
        L[i].res = take((size_t)g.N);
        if (i + 1 < L.size()) {
            const Grid& c = L[i + 1].g;
            L[i].t1 = take((size_t)g.nz * g.ny * c.nx);
            L[i].t2 = take((size_t)g.nz * c.ny * c.nx);
        }
    }
}

void mg_smooth(dft_context* ctx, MGLevel& l, double sscale, int n) {
    for (int s = 0; s < n; ++s) {
        mg_smooth_kernel<<<mg_blocks(ctx, l.g.N), 256, 0, ctx->stream>>>(l.g, l.src, sscale, l.v, l.tmp, 0.8);
        std::swap(l.v, l.tmp);
    }
    count_launch(ctx, n);
}

void vcycle(dft_context* ctx, std::vector<MGLevel>& L, size_t i, double sscale) {
    MGLevel& l = L[i];
    if (i + 1 == L.size()) {
        const size_t sm = sizeof(double) * 2 * (size_t)l.g.N;
        double omega = 1.0;
        int sweeps = 8 * std::max({l.g.nx, l.g.ny, l.g.nz});
        if (ctx->mg_coarsest_sor) coarsest_sor(l.g, &omega, &sweeps);
        mg_coarsest_kernel<<<1, 1024, sm, ctx->stream>>>(l.g, l.src, l.v, sweeps, omega);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        return;
    }
    mg_smooth(ctx, l, sscale, 2);
    mg_residual_kernel<<<mg_blocks(ctx, l.g.N), 256, 0, ctx->stream>>>(l.g, l.src, sscale, l.v, l.res, nullptr);
    count_launch(ctx);
    MGLevel& c = L[i + 1];
    restrict3(ctx, l.g, c.g, l.res, l.t1, l.t2, c.src);
    DFT_CUDA(cudaMemsetAsync(c.v, 0, sizeof(double) * (size_t)c.g.N, ctx->stream));
    vcycle(ctx, L, i + 1, 1.0);
    prolong_add_kernel<<<mg_blocks(ctx, l.g.N), 256, 0, ctx->stream>>>(l.g, c.g, c.v, l.v);
    count_launch(ctx);
    mg_smooth(ctx, l, sscale, 2);
    DFT_LAUNCH_CHECK();
}

}  // namespace

size_t coarse_slab_doubles(const Grid& g) { return slab_doubles(g, plan_levels(g)); }

long coarse_start(dft_context* ctx, double* slab, const Grid& g, const double* rho, double* vup, double** scale_dev) {
    return coarse_solve(ctx, slab, g, rho, vup, scale_dev, nullptr);
}

int multigrid(dft_context* ctx, const Grid& g, const double* rho, double* v, double tol, int max_cycles,
              double* resid_out) {
    std::vector<MGLevel> L = mg_plan(g);
    if (L.back().g.N > MG_COARSEST_MAX) fail(DFT_INVALID_ARGUMENT, "grid too small or too anisotropic for multigrid");
    double* slab = (double*)ws_get(ctx, WS_PG1, sizeof(double) * mg_doubles(L));
    mg_carve(slab, L);
    static bool attr = false;
    if (!attr) {
        DFT_CUDA(cudaFuncSetAttribute(mg_coarsest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(double) * 2 * MG_COARSEST_MAX)));
        attr = true;
    }
    // the fine level works in place on v (its faces must hold the boundary values); rho is
    // its source, scaled by 4 pi
    L[0].src = const_cast<double*>(rho);
    L[0].v = v;
    unsigned long long* rmax = (unsigned long long*)(slab + 8);
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    const double fourpi = 4.0 * 3.14159265358979323846;
    // one cycle: the V-cycle, then the residual's max norm into rmax
    auto cycle = [&] {
        vcycle(ctx, L, 0, fourpi);
        if (L[0].v != v) {  // an odd number of smoothing swaps left the iterate in the temporary
            DFT_CUDA(cudaMemcpyAsync(v, L[0].v, sizeof(double) * (size_t)g.N, cudaMemcpyDeviceToDevice, ctx->stream));
            L[0].tmp = L[0].v;
            L[0].v = v;
        }
        DFT_CUDA(cudaMemsetAsync(rmax, 0, 8, ctx->stream));
        mg_residual_kernel<<<mg_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g, rho, fourpi, v, L[0].res, rmax);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    };
    // The cycle's launch sequence is the same every time for this grid and these buffers: it
    // is captured once as a CUDA graph and replayed (one launch instead of ~10 per level).
    // A capture that fails for any reason leaves the direct launches in place.
    cudaGraphExec_t exec = nullptr;
    long long per_replay = 0;
    if (ctx->multigrid_graphs) {
        const MGGraphKey key{g.nx, g.ny, g.nz, (long long)(uintptr_t)slab, (long long)(uintptr_t)rho,
                             (long long)(uintptr_t)v};
        auto it = ctx->mg_graphs.find(key);
        if (it != ctx->mg_graphs.end()) {
            exec = it->second.exec;
            per_replay = it->second.launches;
        } else {
            const long long l0 = ctx->launches;
            cudaGraph_t graph = nullptr;
            bool captured = false;
            if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                try {
                    cycle();
                } catch (const Error&) {
                }
                captured = cudaStreamEndCapture(ctx->stream, &graph) == cudaSuccess && graph != nullptr;
            }
            cudaGetLastError();  // a failed capture leaves no sticky error; clear the last one
            per_replay = ctx->launches - l0;
            ctx->launches = l0;
            if (captured && L[0].v == v && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
                if (ctx->mg_graphs.size() >= 16) {  // keep a handful: the buffers of the current solves
                    cudaGraphExecDestroy(ctx->mg_graphs.begin()->second.exec);
                    ctx->mg_graphs.erase(ctx->mg_graphs.begin());
                }
                ctx->mg_graphs[key] = {exec, per_replay};
            } else {
                exec = nullptr;
                cudaGetLastError();
            }
            if (graph) cudaGraphDestroy(graph);
        }
    }
    double* h = pinned(ctx, 1);
    int c = 0;
    double r = 0.0;
    for (c = 1; c <= max_cycles; ++c) {
        if (exec) {
            DFT_CUDA(cudaGraphLaunch(exec, ctx->stream));
            count_launch(ctx, per_replay);
        } else {
            cycle();
        }
        DFT_CUDA(cudaMemcpyAsync(h, rmax, 8, cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        r = h[0] / den;  // the size of the next Jacobi update
        if (r < tol) break;
    }
    if (resid_out) *resid_out = r;
    return std::min(c, max_cycles);
}

void poisson_start(dft_context* ctx, dft_pnet* net, const Grid& g, const double* rho, double* out, int cycles,
                   PoissonGuessInfo* info) {
    double* slab = (double*)ws_get(ctx, WS_PG0, sizeof(double) * coarse_slab_doubles(g));
    double* sdev = nullptr;
    const long sw = coarse_start(ctx, slab, g, rho, out, &sdev);
    if (net) pnet_correct(ctx, net, g, rho, out, sdev);
    int used = 0;
    double r = 0.0;
    if (cycles > 0) used = multigrid(ctx, g, rho, out, 0.5e-8, cycles, &r);
    if (info) {
        info->coarse_cycles = sw;
        const Grid gc = coarse_grid(g);
        info->coarse_n[0] = gc.nx;
        info->coarse_n[1] = gc.ny;
        info->coarse_n[2] = gc.nz;
        info->cycles = used;
        info->residual = r;
        double* h = pinned(ctx, 1);
        DFT_CUDA(cudaMemcpyAsync(h, sdev, 8, cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        info->scale = h[0];
    }
}

int synthetic_density(dft_context* ctx, const Grid& g, unsigned long long seed, int kmin, int kmax, double wmin,
                      double wmax, int ne_min, int ne_max, double* rho) {
    if (kmin < 1 || kmax < kmin || kmax > 64 || wmin <= 0 || wmax < wmin || ne_min < 1 || ne_max < ne_min)
        fail(DFT_INVALID_ARGUMENT, "invalid synthetic density parameters");
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> uk(kmin, kmax), une(ne_min, ne_max);
    std::uniform_real_distribution<double> ux(g.xmin, g.xmax), uy(g.ymin, g.ymax), uz(g.zmin, g.zmax),
        uw(wmin, wmax), ua(0.1, 1.0);
    const int k = uk(rng);
    std::vector<Gauss> gs(k);
    for (auto& q : gs) {
        q.x = ux(rng);
        q.y = uy(rng);
        q.z = uz(rng);
        const double w = uw(rng);
        q.inv2w2 = 1.0 / (2.0 * w * w);
        // amplitude per unit charge of a full Gaussian, times a random weight
        q.a = ua(rng) / std::pow(2.0 * 3.14159265358979323846 * w * w, 1.5);
    }
    const int ne = une(rng);
    Gauss* d = (Gauss*)ws_get(ctx, WS_TMP2, sizeof(Gauss) * gs.size());
    DFT_CUDA(cudaMemcpyAsync(d, gs.data(), sizeof(Gauss) * gs.size(), cudaMemcpyHostToDevice, ctx->stream));
    gauss_density_kernel<<<blocks_for(ctx, g.N), 256, 0, ctx->stream>>>(g, d, k, rho);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    double* tot = (double*)ws_get(ctx, WS_TMP, sizeof(double));
    sum_kernel<<<1, 1024, 0, ctx->stream>>>(g.N, rho, tot);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    double* h = pinned(ctx, 1);
    DFT_CUDA(cudaMemcpyAsync(h, tot, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);  // also keeps gs alive until the density kernel has read it
    const double q = h[0] * g.dV;
    if (!(q > 0.0)) fail(DFT_NUMERICAL, "synthetic density has no charge on the grid");
    scale_kernel<<<blocks_for(ctx, g.N), 256, 0, ctx->stream>>>(g.N, rho, (double)ne / q);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    return ne;
}


}  // namespace dftb
