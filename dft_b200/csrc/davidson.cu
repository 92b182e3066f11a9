// Block Davidson eigensolver for H = -1/2 lap_h + V on the device.
//
// The reference solves one orbital at a time with a single-vector Davidson, deflating each
// new orbital against all previous ones (EigenvalueSolverMolecule.cpp:666-1300).  That
// costs O(i N) vector passes per step for orbital i and runs one H psi at a time.  Here all
// nbands bands advance together:
//
//   basis V (orthonormal, dV-weighted), AV = H V
//   G = dV V^T AV  -> eigh(G) -> Ritz pairs (theta, Y) for the lowest nbands
//   X = V Y, AX = AV Y, R = AX - X theta, |r_b| = sqrt(dV sum R_b^2)
//   occupied bands converge at |r_b| < tol (reference MO_RESIDUAL_TOLERANCE = 1e-7)
//   T = R_b / (theta_b - diag) for unconverged bands (the reference's davidsonCorrection,
//       :521-555, with the same 1e-10 guard), projected out of V twice and orthonormalised
//       by the symmetric (SVQB) scheme, then appended; thick restart to [X] when full.
//
// Tall-skinny products (Gram V^T W, rotation V Y) are FP64 kernels with warp/block
// reductions; the k x k eigenproblems are solved on the host (eigh.cpp).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "eigh.h"
#include "neural.h"
#include "ops.h"

namespace dftb {

namespace {

// ------------------------------------------------------------------ kernels ----------

// buildInitialVector (reference EigenvalueSolverMolecule.cpp:177-283) for seeds seed0+b.
__global__ void seed_kernel(Grid g, double* psi, long long ld, int nb, int seed0) {
    const int b = blockIdx.y;
    const int idx = seed0 + b;
    const double cx = 0.5 * (g.xmin + g.xmax), cy = 0.5 * (g.ymin + g.ymax), cz = 0.5 * (g.zmin + g.zmax);
    const double sigma = 0.8 + 0.18 * (double)idx;
    const double factor = 1.0 / (2.0 * sigma * sigma);
    const int mode = idx % 9;
    double* out = psi + (long long)b * ld;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx);
        const int j = (int)((p / g.nx) % g.ny);
        const int k = (int)(p / ((long long)g.nx * g.ny));
        const double x = __dadd_rn(g.xmin, __dmul_rn((double)i, g.dx)) - cx;
        const double y = __dadd_rn(g.ymin, __dmul_rn((double)j, g.dy)) - cy;
        const double z = __dadd_rn(g.zmin, __dmul_rn((double)k, g.dz)) - cz;
        const double r2 = x * x + y * y + z * z;
        double pl = 1.0;
        switch (mode) {
            case 1: pl = x; break;
            case 2: pl = y; break;
            case 3: pl = z; break;
            case 4: pl = x * y; break;
            case 5: pl = x * z; break;
            case 6: pl = y * z; break;
            case 7: pl = x * x - y * y; break;
            case 8: pl = 2.0 * z * z - x * x - y * y; break;
            default: break;
        }
        out[p] = pl * exp(-r2 * factor);
    }
}

constexpr int GT = 32;          // Gram output tile (GT x GT)
constexpr int GP = 32;          // points per shared-memory stage
constexpr int GRAM_THREADS = 256;

// partial[c][i][j] = sum over chunk c of A_i[p] B_j[p] for one GT x GT output tile.
// 256 threads = 16 x 16, each owns a 2 x 2 block of the tile.
__global__ void __launch_bounds__(GRAM_THREADS) gram_kernel(const double* __restrict__ A, long long lda, int ka,
                                                            const double* __restrict__ B, long long ldb, int kb,
                                                            long long n, long long chunk, double* __restrict__ partial) {
    __shared__ double sa[GT][GP + 1];
    __shared__ double sb[GT][GP + 1];
    const int ti = blockIdx.x * GT, tj = blockIdx.y * GT;
    const long long p0 = (long long)blockIdx.z * chunk;
    const long long p1 = min(n, p0 + chunk);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc00 = 0.0, acc01 = 0.0, acc10 = 0.0, acc11 = 0.0;
    for (long long ps = p0; ps < p1; ps += GP) {
        // stage GT vectors x GP points of A and B (coalesced along points)
        for (int e = threadIdx.x; e < GT * GP; e += GRAM_THREADS) {
            const int r = e / GP, c = e % GP;
            const long long p = ps + c;
            const int ia = ti + r, jb = tj + r;
            sa[r][c] = (ia < ka && p < p1) ? A[(long long)ia * lda + p] : 0.0;
            sb[r][c] = (jb < kb && p < p1) ? B[(long long)jb * ldb + p] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int c = 0; c < GP; ++c) {
            const double a0 = sa[ty][c], a1 = sa[ty + 16][c];
            const double b0 = sb[tx][c], b1 = sb[tx + 16][c];
            acc00 += a0 * b0;
            acc01 += a0 * b1;
            acc10 += a1 * b0;
            acc11 += a1 * b1;
        }
        __syncthreads();
    }
    double* out = partial + (long long)blockIdx.z * ka * kb;
    const int i0 = ti + ty, i1 = ti + ty + 16, j0 = tj + tx, j1 = tj + tx + 16;
    if (i0 < ka && j0 < kb) out[(long long)i0 * kb + j0] = acc00;
    if (i0 < ka && j1 < kb) out[(long long)i0 * kb + j1] = acc01;
    if (i1 < ka && j0 < kb) out[(long long)i1 * kb + j0] = acc10;
    if (i1 < ka && j1 < kb) out[(long long)i1 * kb + j1] = acc11;
}

// out[e] = scale * sum_c partial[c][e]: one warp per element, lanes stride the chunks, fixed
// shuffle order (deterministic)
__global__ void gram_reduce_kernel(int nchunks, int nel, const double* __restrict__ partial, double scale,
                                   double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    for (int e = blockIdx.x * warps + (threadIdx.x >> 5); e < nel; e += gridDim.x * warps) {
        double s = 0.0;
        for (int c = lane; c < nchunks; c += 32) s += partial[(long long)c * nel + e];
        s = warp_sum(s);
        if (lane == 0) out[e] = s * scale;
    }
}

constexpr int RJ = 16;  // output columns per rotation block

// out_j = beta*out_j + alpha * sum_i in_i * Y[i*m + j], j in a RJ-column slice per blockIdx.y
__global__ void __launch_bounds__(256) rotate_kernel(const double* __restrict__ in, long long ldi, int k,
                                                     const double* __restrict__ Y, int m, double* __restrict__ out,
                                                     long long ldo, long long n, double alpha, double beta) {
    extern __shared__ double sy[];  // k x RJ
    const int j0 = blockIdx.y * RJ;
    const int nj = min(RJ, m - j0);
    for (int e = threadIdx.x; e < k * RJ; e += blockDim.x) {
        const int i = e / RJ, jj = e % RJ;
        sy[e] = jj < nj ? Y[(long long)i * m + j0 + jj] : 0.0;
    }
    __syncthreads();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        double acc[RJ];
#pragma unroll
        for (int jj = 0; jj < RJ; ++jj) acc[jj] = 0.0;
        for (int i = 0; i < k; ++i) {
            const double v = __ldg(in + (long long)i * ldi + p);
#pragma unroll
            for (int jj = 0; jj < RJ; ++jj) acc[jj] += v * sy[i * RJ + jj];
        }
#pragma unroll
        for (int jj = 0; jj < RJ; ++jj) {
            if (jj < nj) {
                double* o = out + (long long)(j0 + jj) * ldo + p;
                *o = beta == 0.0 ? alpha * acc[jj] : beta * *o + alpha * acc[jj];
            }
        }
    }
}

// R_b = AX_b - theta_b X_b and per-block partial sums of R_b^2 (blockIdx.y = band)
__global__ void __launch_bounds__(256) residual_kernel(const double* __restrict__ AX, const double* __restrict__ X,
                                                       const double* __restrict__ theta, double* __restrict__ R,
                                                       long long ld, long long n, double* __restrict__ partial) {
    __shared__ double sh[8];
    const int b = blockIdx.y;
    const double t = theta[b];
    const double* ax = AX + (long long)b * ld;
    const double* x = X + (long long)b * ld;
    double* r = R + (long long)b * ld;
    double s = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double v = ax[p] - t * x[p];
        r[p] = v;
        s += v * v;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[(long long)b * gridDim.x + blockIdx.x] = s;
}

// T_a = R_src(a) / (theta - (kin + V)) with the reference guard (|den| < 1e-10 or non-finite
// -> T = R), reference davidsonCorrection :521-555, buildHamiltonianDiagonal :483-519.
__global__ void precond_kernel(const double* __restrict__ R, const double* __restrict__ V, const int* __restrict__ src,
                               const double* __restrict__ theta, double* __restrict__ T, long long ld, long long n,
                               double kin) {
    const int a = blockIdx.y;
    const int b = src[a];
    const double t = theta[b];
    const double* r = R + (long long)b * ld;
    double* o = T + (long long)a * ld;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double den = t - (kin + V[p]);
        o[p] = (!isfinite(den) || fabs(den) < 1.0e-10) ? r[p] : r[p] / den;
    }
}

// Kinetic preconditioner step: one damped-Jacobi step for (T + sigma_a) t = r_a, T = -1/2 lap_h
// with psi = 0 outside the box.  out = (1-w) t + w (r + 1/2 S(t)) / (kin + sigma_a), where S is
// the weighted sum of the six neighbours; t == nullptr means t = 0 (then out = w r / d).
// Smooths the high-frequency (large kinetic energy) part of the residual, which the reference's
// diagonal preconditioner leaves almost untouched on fine grids.
__global__ void __launch_bounds__(256) kinetic_smooth_kernel(Grid g, const double* __restrict__ t,
                                                             const double* __restrict__ R, const int* __restrict__ src,
                                                             const double* __restrict__ sigma, double* __restrict__ out,
                                                             long long ld, int zchunk, int nzc, double w) {
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    const int a = blockIdx.z / nzc;
    const int kc = blockIdx.z - a * nzc;
    if (i >= g.nx || j >= g.ny) return;
    const double* __restrict__ r = R + (long long)src[a] * ld;
    const double* __restrict__ tp = t ? t + (long long)a * ld : nullptr;
    double* __restrict__ o = out + (long long)a * ld;
    const double d = g.ix2 + g.iy2 + g.iz2 + sigma[a];
    const long long sxy = (long long)g.nx * g.ny;
    const int kb = kc * zchunk, ke = min(g.nz, kb + zchunk);
    long long idx = (long long)kb * sxy + (long long)j * g.nx + i;
    if (!tp) {
        for (int k = kb; k < ke; ++k, idx += sxy) o[idx] = w * r[idx] / d;
        return;
    }
    double below = kb > 0 ? tp[idx - sxy] : 0.0, cur = tp[idx];
    for (int k = kb; k < ke; ++k, idx += sxy) {
        const double above = k + 1 < g.nz ? tp[idx + sxy] : 0.0;
        double s = g.iz2 * (below + above);
        if (i > 0) s += g.ix2 * tp[idx - 1];
        if (i + 1 < g.nx) s += g.ix2 * tp[idx + 1];
        if (j > 0) s += g.iy2 * tp[idx - g.nx];
        if (j + 1 < g.ny) s += g.iy2 * tp[idx + g.nx];
        o[idx] = (1.0 - w) * cur + w * (r[idx] + 0.5 * s) / d;
        below = cur;
        cur = above;
    }
}

__global__ void rows_sum_kernel2(int nrows, int ncols, const double* partial, double* out) {
    __shared__ double sh[32];
    for (int r = 0; r < nrows; ++r) {
        double s = 0.0;
        for (int c = threadIdx.x; c < ncols; c += blockDim.x) s += partial[(long long)r * ncols + c];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) out[r] = s;
    }
}

// ------------------------------------------------------------------ host helpers -----

struct Blocks {
    dft_context* ctx;
    Grid g;
    long long ld;
};

// Narrow Gram products (ka <= 64, kb <= KB): one launch.  Warp w of every block owns rows
// i = w, w + 8, ... of A (RPW of them) and all kb columns; its lanes stride the points and
// keep RPW x KB sums in registers.  Block partials go to `partial`; the partials are then
// added in two fixed-order levels inside the same launch: the last block to finish in each
// group of GS_GROUP blocks (ticket[1 + group]) adds its group's partials, and the last group
// to finish (ticket[0]) adds the group sums and writes dV * C.  Every thread of a reducing
// block owns whole elements and issues its (at most GS_GROUP) loads at once, so the tail is a
// few L2 round trips instead of one dependent chain per element.
constexpr int GS_GROUP = 16;
constexpr int GS_TICKETS = 256;  // ticket words: 1 + groups (blocks <= 4 x SMs)

template <int RPW, int KB>
__global__ void __launch_bounds__(256) gram_small_kernel(const double* __restrict__ A, long long lda, int ka,
                                                         const double* __restrict__ B, long long ldb, int kb,
                                                         long long n, double scale, double* __restrict__ partial,
                                                         unsigned int* __restrict__ ticket, double* __restrict__ out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc[RPW][KB];
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int j = 0; j < KB; ++j) acc[r][j] = 0.0;
    // two points per step (both loads issued before the FMAs) for more loads in flight
    const long long stride = (long long)gridDim.x * 32;
    for (long long p = (long long)blockIdx.x * 32 + lane; p < n; p += 2 * stride) {
        const long long p2 = p + stride;
        const bool has2 = p2 < n;
        double b[KB], b2[KB];
#pragma unroll
        for (int j = 0; j < KB; ++j) {
            b[j] = j < kb ? __ldg(B + (long long)j * ldb + p) : 0.0;
            b2[j] = (j < kb && has2) ? __ldg(B + (long long)j * ldb + p2) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < RPW; ++r) {
            const int i = warp + 8 * r;
            const double a = i < ka ? __ldg(A + (long long)i * lda + p) : 0.0;
            const double a2 = (i < ka && has2) ? __ldg(A + (long long)i * lda + p2) : 0.0;
#pragma unroll
            for (int j = 0; j < KB; ++j) acc[r][j] = fma(a2, b2[j], fma(a, b[j], acc[r][j]));
        }
    }
    const int nel = ka * kb;
    double* mine = partial + (long long)blockIdx.x * nel;
#pragma unroll
    for (int r = 0; r < RPW; ++r)
#pragma unroll
        for (int j = 0; j < KB; ++j) {
            const double v = warp_sum(acc[r][j]);
            const int i = warp + 8 * r;
            if (lane == 0 && i < ka && j < kb) mine[i * kb + j] = v;
        }
    // level 1: the last block of this group adds the group's partials in block order
    const int nblk = (int)gridDim.x;
    const int ngroups = (nblk + GS_GROUP - 1) / GS_GROUP;
    const int grp = (int)blockIdx.x / GS_GROUP;
    const int g0 = grp * GS_GROUP;
    const int gsz = min(GS_GROUP, nblk - g0);
    double* gsum = partial + (long long)nblk * nel;  // [ngroups][nel]
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket + 1 + grp, 1u) == (unsigned)gsz - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
        double v[GS_GROUP];
#pragma unroll
        for (int c = 0; c < GS_GROUP; ++c) v[c] = c < gsz ? __ldcg(partial + (long long)(g0 + c) * nel + e) : 0.0;
        double sum = 0.0;
#pragma unroll
        for (int c = 0; c < GS_GROUP; ++c) sum += v[c];
        gsum[(long long)grp * nel + e] = sum;
    }
    if (threadIdx.x == 0) ticket[1 + grp] = 0;  // ready for the next call
    // level 2: the last group adds the group sums in group order
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == (unsigned)ngroups - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int e = threadIdx.x; e < nel; e += blockDim.x) {
        double sum = 0.0;
        for (int c0 = 0; c0 < ngroups; c0 += 8) {
            double v[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) v[c] = c0 + c < ngroups ? __ldcg(gsum + (long long)(c0 + c) * nel + e) : 0.0;
#pragma unroll
            for (int c = 0; c < 8; ++c) sum += v[c];
        }
        out[e] = sum * scale;
    }
    if (threadIdx.x == 0) *ticket = 0;
}

// C (ka x kb, host, row-major) = dV * A^T B
void gram(dft_context* ctx, const Grid& g, const double* A, long long lda, int ka, const double* B, long long ldb,
          int kb, std::vector<double>& C) {
    C.assign((size_t)ka * kb, 0.0);
    if (ka == 0 || kb == 0) return;
    const int rpw = ka <= 8 ? 1 : ka <= 16 ? 2 : ka <= 32 ? 4 : 8;
    const int kbt = kb <= 4 ? 4 : kb <= 8 ? 8 : 16;
    if (ka <= 64 && kb <= 16 && rpw * kbt <= 64) {
        // narrow product: one launch, the last block reduces
        const size_t nel = (size_t)ka * kb;
        const int nblk = (int)std::max<long long>(
            1, std::min<long long>(std::min(4LL * ctx->num_sms, (long long)(GS_TICKETS - 1) * GS_GROUP),
                                   (g.N + 255) / 256));
        const int ngroups = (nblk + GS_GROUP - 1) / GS_GROUP;
        double* partial = (double*)ws_get(ctx, WS_SMALL, sizeof(double) * (nel * (nblk + ngroups) + nel) + 64);
        double* res = partial + nel * (nblk + ngroups);
        if (!ctx->gram_ticket) {
            DFT_CUDA(cudaMalloc(&ctx->gram_ticket, sizeof(unsigned int) * GS_TICKETS));
            DFT_CUDA(cudaMemsetAsync(ctx->gram_ticket, 0, sizeof(unsigned int) * GS_TICKETS, ctx->stream));
        }
        unsigned int* tk = (unsigned int*)ctx->gram_ticket;
#define DFT_GS(R, K)                                                                                          \
    gram_small_kernel<R, K><<<nblk, 256, 0, ctx->stream>>>(A, lda, ka, B, ldb, kb, g.N, g.dV, partial, tk, res)
        switch (rpw * 100 + kbt) {
            case 104: DFT_GS(1, 4); break;
            case 108: DFT_GS(1, 8); break;
            case 116: DFT_GS(1, 16); break;
            case 204: DFT_GS(2, 4); break;
            case 208: DFT_GS(2, 8); break;
            case 216: DFT_GS(2, 16); break;
            case 404: DFT_GS(4, 4); break;
            case 408: DFT_GS(4, 8); break;
            case 416: DFT_GS(4, 16); break;
            case 804: DFT_GS(8, 4); break;
            default: DFT_GS(8, 8); break;
        }
#undef DFT_GS
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        double* h = pinned(ctx, nel);
        DFT_CUDA(cudaMemcpyAsync(h, res, sizeof(double) * nel, cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        std::memcpy(C.data(), h, sizeof(double) * nel);
        return;
    }
    const int tx = (ka + GT - 1) / GT, ty = (kb + GT - 1) / GT;
    long long target = 4LL * ctx->num_sms;
    long long nch = std::max<long long>(1, target / (tx * ty));
    long long chunk = (g.N + nch - 1) / nch;
    chunk = ((chunk + GP - 1) / GP) * GP;
    nch = (g.N + chunk - 1) / chunk;
    nch = std::min<long long>(nch, 65535);
    chunk = (g.N + nch - 1) / nch;
    const size_t nel = (size_t)ka * kb;
    double* partial = (double*)ws_get(ctx, WS_SMALL, sizeof(double) * (nel * nch + nel));
    double* res = partial + nel * nch;
    gram_kernel<<<dim3(tx, ty, (unsigned)nch), GRAM_THREADS, 0, ctx->stream>>>(A, lda, ka, B, ldb, kb, g.N, chunk,
                                                                               partial);
    DFT_LAUNCH_CHECK();
    const int rb = (int)std::min<size_t>((nel + 7) / 8, 4096);  // 8 warps per block, one element per warp
    gram_reduce_kernel<<<rb, 256, 0, ctx->stream>>>((int)nch, (int)nel, partial, g.dV, res);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    double* h = pinned(ctx, nel);
    DFT_CUDA(cudaMemcpyAsync(h, res, sizeof(double) * nel, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    std::memcpy(C.data(), h, sizeof(double) * nel);
}

}  // namespace

// out = beta*out + alpha * in * Y   (Y: k x m host row-major)
void rotate(dft_context* ctx, const Grid& g, const double* in, long long ldi, int k, const std::vector<double>& Y, int m,
            double* out, long long ldo, double alpha, double beta) {
    if (m == 0) return;
    if (k == 0) {
        if (beta == 0.0)
            for (int j = 0; j < m; ++j)
                DFT_CUDA(cudaMemsetAsync(out + (long long)j * ldo, 0, sizeof(double) * (size_t)g.N, ctx->stream));
        return;
    }
    double* dy = (double*)ws_get(ctx, WS_TMP, sizeof(double) * (size_t)k * m);
    DFT_CUDA(cudaMemcpyAsync(dy, Y.data(), sizeof(double) * (size_t)k * m, cudaMemcpyHostToDevice, ctx->stream));
    const int jt = (m + RJ - 1) / RJ;
    const size_t smem = sizeof(double) * (size_t)k * RJ;
    if (smem > 200 * 1024) fail(DFT_INVALID_ARGUMENT, "subspace too large for the rotation kernel (k=%d)", k);
    static bool attr_set = false;
    if (!attr_set) {
        DFT_CUDA(cudaFuncSetAttribute(rotate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_set = true;
    }
    long long bx = (g.N + 255) / 256;
    bx = std::min<long long>(bx, std::max<long long>(1, (8LL * ctx->num_sms + jt - 1) / jt));
    rotate_kernel<<<dim3((unsigned)bx, jt), 256, smem, ctx->stream>>>(in, ldi, k, dy, m, out, ldo, g.N, alpha, beta);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

namespace {

// Y = L^-T for the Cholesky factor S = L L^T of an n x n SPD matrix (row-major), so that
// T Y has the identity as Gram matrix.  False when a pivot falls below rel * max diag(S).
bool cholesky_inverse_t(int n, const std::vector<double>& S, double rel, std::vector<double>& Y) {
    double smax = 0.0;
    for (int i = 0; i < n; ++i) smax = std::max(smax, S[(size_t)i * n + i]);
    if (!(smax > 0.0) || !std::isfinite(smax)) return false;
    std::vector<double> L((size_t)n * n, 0.0);
    for (int j = 0; j < n; ++j) {
        double d = S[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
        if (!(d > rel * smax)) return false;
        const double ljj = std::sqrt(d);
        L[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            double v = S[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) v -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            L[(size_t)i * n + j] = v / ljj;
        }
    }
    // M = L^-1 (lower triangular) by forward substitution, column by column; Y = M^T
    Y.assign((size_t)n * n, 0.0);
    for (int c = 0; c < n; ++c) {
        for (int i = c; i < n; ++i) {
            double v = i == c ? 1.0 : 0.0;
            for (int k = c; k < i; ++k) v -= L[(size_t)i * n + k] * Y[(size_t)c * n + k];
            Y[(size_t)c * n + i] = v / L[(size_t)i * n + i];  // Y[c][i] = M[i][c]
        }
    }
    for (double v : Y)
        if (!std::isfinite(v)) return false;
    return true;
}

// Orthonormalise the nt columns of T against V[0:k] and among themselves (dV inner product).
// Dependent directions are dropped; returns the number kept (compacted to the front of T).
// tc: Gram products on the tensor cores (TF32 hi+lo, ~1e-6 relative) instead of FP64
void gram_any(bool tc, dft_context* ctx, const Grid& g, const double* A, long long lda, int ka, const double* B,
              long long ldb, int kb, std::vector<double>& C) {
    // the tensor-core product pays only when both blocks are wide enough to fill its tiles;
    // narrow products (few bands) are latency-bound either way and stay in FP64
    if (tc && (long long)ka * kb >= 2048) gram_tc(ctx, g, A, lda, ka, B, ldb, kb, C);
    else gram(ctx, g, A, lda, ka, B, ldb, kb, C);
}

int orthonormalise(dft_context* ctx, const Grid& g, const double* V, int k, double* T, int nt, long long ld,
                   double* W, bool tc = false) {
    std::vector<double> C, S, w, Z, Yk;
    // directions below the Gram products' noise floor are dropped
    const double floor_rel = tc ? 1e-8 : 1e-13;
    const double chol_rel = tc ? 1e-7 : 1e-12;
    for (int pass = 0; pass < 2 && nt > 0; ++pass) {
        if (k > 0 && T == V + (long long)k * ld) {
            // one product [V; T]^T T gives C = V^T T and T^T T; the projected block's Gram is then
            // T^T T - C^T C, and one rotation applies T <- (T - V C) L^-T (V orthonormal)
            std::vector<double> M;
            gram_any(tc, ctx, g, V, ld, k + nt, T, ld, nt, M);  // (k + nt) x nt
            S.assign((size_t)nt * nt, 0.0);
            for (int i = 0; i < nt; ++i)
                for (int j = 0; j <= i; ++j) {
                    double v = 0.5 * (M[(size_t)(k + i) * nt + j] + M[(size_t)(k + j) * nt + i]);
                    for (int r = 0; r < k; ++r) v -= M[(size_t)r * nt + i] * M[(size_t)r * nt + j];
                    S[(size_t)i * nt + j] = S[(size_t)j * nt + i] = v;
                }
            if (cholesky_inverse_t(nt, S, chol_rel, Yk)) {
                std::vector<double> Yc((size_t)(k + nt) * nt, 0.0);
                for (int r = 0; r < k; ++r)
                    for (int j = 0; j < nt; ++j) {
                        double v = 0.0;
                        for (int c = 0; c <= j; ++c) v -= M[(size_t)r * nt + c] * Yk[(size_t)c * nt + j];
                        Yc[(size_t)r * nt + j] = v;
                    }
                for (int i = 0; i < nt; ++i)
                    for (int j = 0; j < nt; ++j) Yc[(size_t)(k + i) * nt + j] = Yk[(size_t)i * nt + j];
                // in mixed-precision mode a wide rotation runs on the tensor cores like the Ritz
                // rotations (the second pass restores orthonormality to the products' accuracy)
                if (tc && k + nt >= 32 && (long long)(k + nt) * nt >= 2048)
                    rotate_tc(ctx, g, V, ld, k + nt, Yc, nt, W, ld);
                else
                    rotate(ctx, g, V, ld, k + nt, Yc, nt, W, ld, 1.0, 0.0);
                DFT_CUDA(cudaMemcpyAsync(T, W, sizeof(double) * (size_t)ld * nt, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
                // In FP64 one pass suffices when the block was far from dependent: the loss of
                // orthogonality of projected Cholesky QR is about eps * r * kappa(S), with
                // r = max_i (T^T T)_ii / S_ii (the cancellation of the projection) and
                // kappa(S) <= trace(S) ||L^-T||_F^2.  Below 1e-12 the second pass is skipped.
                if (!tc && pass == 0 && ctx->ortho_adaptive) {
                    double r = 1.0, tr = 0.0, yf = 0.0;
                    for (int i = 0; i < nt; ++i) {
                        const double sii = S[(size_t)i * nt + i];
                        r = std::max(r, M[(size_t)(k + i) * nt + i] / sii);
                        tr += sii;
                    }
                    for (double v : Yk) yf += v * v;
                    const double est = 2.2204460492503131e-16 * 16.0 * r * tr * yf;
                    if (std::isfinite(est) && est < 1e-12) break;
                }
                continue;
            }
            // nearly dependent: project with the C already at hand, then the explicit path below
            C.assign((size_t)k * nt, 0.0);
            for (size_t q = 0; q < (size_t)k * nt; ++q) C[q] = M[q];
            rotate(ctx, g, V, ld, k, C, nt, T, ld, -1.0, 1.0);
        } else if (k > 0) {
            gram_any(tc, ctx, g, V, ld, k, T, ld, nt, C);  // k x nt
            rotate(ctx, g, V, ld, k, C, nt, T, ld, -1.0, 1.0);
        }
        gram_any(tc, ctx, g, T, ld, nt, T, ld, nt, S);
        for (int i = 0; i < nt; ++i)
            for (int j = 0; j < i; ++j) S[(size_t)i * nt + j] = S[(size_t)j * nt + i] = 0.5 * (S[(size_t)i * nt + j] + S[(size_t)j * nt + i]);
        // Cholesky QR: S = L L^T, T <- T L^-T, when every pivot stays well above round-off
        // (O(nt^3/3) on the host); a nearly dependent block falls through to the SVQB below,
        // which drops the dependent directions
        if (cholesky_inverse_t(nt, S, chol_rel, Yk)) {
            rotate(ctx, g, T, ld, nt, Yk, nt, W, ld, 1.0, 0.0);
            DFT_CUDA(cudaMemcpyAsync(T, W, sizeof(double) * (size_t)ld * nt, cudaMemcpyDeviceToDevice, ctx->stream));
            continue;
        }
        std::vector<double> Sc = S;
        if (!eigh(nt, Sc, w, Z)) fail(DFT_NUMERICAL, "orthonormalisation eigensolve failed");
        const double wmax = w[nt - 1];
        if (!(wmax > 0.0) || !std::isfinite(wmax)) return 0;
        // keep eigen-directions well above round-off; scale by lambda^{-1/2}
        std::vector<int> keep;
        for (int j = 0; j < nt; ++j)
            if (w[j] > wmax * floor_rel && w[j] > 1e-24) keep.push_back(j);
        const int nk = (int)keep.size();
        Yk.assign((size_t)nt * nk, 0.0);
        for (int i = 0; i < nt; ++i)
            for (int c = 0; c < nk; ++c) Yk[(size_t)i * nk + c] = Z[(size_t)i * nt + keep[c]] / std::sqrt(w[keep[c]]);
        rotate(ctx, g, T, ld, nt, Yk, nk, W, ld, 1.0, 0.0);
        DFT_CUDA(cudaMemcpyAsync(T, W, sizeof(double) * (size_t)ld * nk, cudaMemcpyDeviceToDevice, ctx->stream));
        nt = nk;
    }
    return nt;
}

}  // namespace

void gram_fp64(dft_context* ctx, const Grid& g, const double* A, long long lda, int ka, const double* B,
               long long ldb, int kb, std::vector<double>& C) {
    gram(ctx, g, A, lda, ka, B, ldb, kb, C);
}

int solve_orbitals(dft_context* ctx, const Grid& g, const double* V, int nocc, int nbands, double* psi,
                   long long ld, bool init, double* eig_host, double* resid_host, const EigOpts& o,
                   const double* start, int nstart) {
    if (nocc <= 0) fail(DFT_INVALID_ARGUMENT, "El numero de orbitales debe ser mayor que cero.");
    if (nbands < nocc) fail(DFT_INVALID_ARGUMENT, "nbands must be >= the number of orbitals");
    if (nbands > g.N) fail(DFT_INVALID_ARGUMENT, "more bands than grid points");
    if (ld < g.N) fail(DFT_INVALID_ARGUMENT, "ld must be >= nx*ny*nz");
    if (o.precond_steps == -3 && !o.precond_net) fail(DFT_INVALID_ARGUMENT, "preconditioner -3 needs a network");
    if (o.precond_steps < -3) fail(DFT_INVALID_ARGUMENT, "unknown preconditioner %d", o.precond_steps);
    const int nb = nbands;
    // basis cap: max_subspace x nbands, and at least nbands + 16 (the reference's subspace of 16);
    // a restart keeps the lowest kr Ritz vectors (thick restart)
    long long km = std::max<long long>(o.max_subspace * (long long)nb, nb + 16LL);
    km = std::max<long long>(km, 2LL * nb);
    const int kmax = (int)std::min<long long>(km, g.N);
    const int kr = std::max(nb, std::min(kmax - 1, kmax / 2));
    const size_t vecb = sizeof(double) * (size_t)ld;
    double* Vb = (double*)ws_get(ctx, WS_DAV0, vecb * kmax);
    double* AV = (double*)ws_get(ctx, WS_DAV1, vecb * kmax);
    double* X = (double*)ws_get(ctx, WS_DAV2, vecb * nb);
    double* AX = (double*)ws_get(ctx, WS_DAV3, vecb * nb);
    double* R = (double*)ws_get(ctx, WS_DAV4, vecb * nb);
    double* W = (double*)ws_get(ctx, WS_DAV5, vecb * std::max(nb, kr));
    const double kin = g.ix2 + g.iy2 + g.iz2;  // buildHamiltonianDiagonal :496-500 (1/dx^2 + 1/dy^2 + 1/dz^2)
    const int eb = std::max(1, std::min((int)((g.N + 255) / 256), ctx->num_sms * 2));

    // ---- start block: a given start basis, given vectors or the reference's seeds -------
    int k0 = nb;
    if (start && nstart > 0) {
        // a start basis of any width (e.g. atomic orbitals): the first Rayleigh-Ritz step picks
        // the lowest nb combinations
        k0 = std::min(nstart, kmax - 1);
        DFT_CUDA(cudaMemcpy2DAsync(Vb, vecb, start, vecb, sizeof(double) * (size_t)g.N, k0, cudaMemcpyDeviceToDevice,
                                   ctx->stream));
        if (k0 > std::max(nb, kr)) W = (double*)ws_get(ctx, WS_DAV5, vecb * k0);
    } else if (init) {
        DFT_CUDA(cudaMemcpy2DAsync(Vb, vecb, psi, vecb, sizeof(double) * (size_t)g.N, nb, cudaMemcpyDeviceToDevice,
                                   ctx->stream));
    } else {
        seed_kernel<<<dim3(eb, nb), 256, 0, ctx->stream>>>(g, Vb, ld, nb, 0);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
    int k = orthonormalise(ctx, g, Vb, 0, Vb, k0, ld, W);
    int seed = nb;
    while (k < nb) {  // rank-deficient start: top up with further seeds
        const int need = nb - k;
        seed_kernel<<<dim3(eb, need), 256, 0, ctx->stream>>>(g, Vb + (long long)k * ld, ld, need, seed);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        seed += need;
        const int got = orthonormalise(ctx, g, Vb, k, Vb + (long long)k * ld, need, ld, W);
        k += got;
        if (seed > nb + 512) fail(DFT_NOT_CONVERGED, "No se pudo construir el vector inicial.");
    }
    apply_hamiltonian(ctx, g, V, Vb, AV, k, ld);

    // Mixed precision: while the occupied residuals are above mixed_switch the Gram products run
    // on the tensor cores (TF32 hi+lo); then the basis restarts from the Ritz block in FP64 and
    // every later product (and the convergence test) is FP64.
    bool tc_mode = o.mixed_precision != 0;
    double tc_best = INFINITY;  // best occupied residual seen in tensor-core mode, and when
    int tc_best_it = 0;
    std::vector<double> G;  // k x k, row-major, grows
    auto grow_G = [&](int k_old, int k_new) {
        std::vector<double> Gn((size_t)k_new * k_new, 0.0);
        for (int i = 0; i < k_old; ++i)
            for (int j = 0; j < k_old; ++j) Gn[(size_t)i * k_new + j] = G[(size_t)i * k_old + j];
        std::vector<double> C;
        gram_any(tc_mode, ctx, g, Vb, ld, k_new, AV + (long long)k_old * ld, ld, k_new - k_old, C);
        const int nn = k_new - k_old;
        for (int i = 0; i < k_new; ++i)
            for (int c = 0; c < nn; ++c) {
                const int j = k_old + c;
                const double v = C[(size_t)i * nn + c];
                if (i >= k_old && i < j) continue;  // set from the symmetric partner below
                Gn[(size_t)i * k_new + j] = v;
                Gn[(size_t)j * k_new + i] = v;
            }
        // symmetrise the new diagonal block
        for (int a = k_old; a < k_new; ++a)
            for (int b2 = k_old; b2 < a; ++b2) {
                const double v = 0.5 * (C[(size_t)a * nn + (b2 - k_old)] + C[(size_t)b2 * nn + (a - k_old)]);
                Gn[(size_t)a * k_new + b2] = Gn[(size_t)b2 * k_new + a] = v;
            }
        G.swap(Gn);
    };
    grow_G(0, k);

    // out = in * Y: on the tensor cores in mixed-precision mode when the block is wide enough
    auto rot = [&](const double* in, int kin, const std::vector<double>& Ym, int m, double* out) {
        if (tc_mode && kin >= 32 && (long long)kin * m >= 2048) rotate_tc(ctx, g, in, ld, kin, Ym, m, out, ld);
        else rotate(ctx, g, in, ld, kin, Ym, m, out, ld, 1.0, 0.0);
    };
    double* dtheta = (double*)ws_get(ctx, WS_DAV6, sizeof(double) * 2 * nb + sizeof(int) * nb + 64);
    double* dsigma = dtheta + nb;
    int* dsrc = (int*)(dsigma + nb);
    std::vector<double> theta(nb), rn(nb), w, Z, Y;
    std::vector<int> active;
    int it = 0;
    bool done = false;
    for (it = 1; it <= o.max_iterations; ++it) {
        // ---- Rayleigh–Ritz --------------------------------------------------------------
        // the lowest nb Ritz pairs only (Z: k x nb); a thick restart below asks for more
        std::vector<double> Gc = G;
        if (!eigh_lowest(k, Gc, nb, w, Z)) fail(DFT_NUMERICAL, "projected eigensolve failed");
        Y = Z;
        for (int j = 0; j < nb; ++j) theta[j] = w[j];
        rot(Vb, k, Y, nb, X);
        rot(AV, k, Y, nb, AX);
        // ---- residuals --------------------------------------------------------------------
        DFT_CUDA(cudaMemcpyAsync(dtheta, theta.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, ctx->stream));
        double* partial = (double*)ws_get(ctx, WS_REDUCE, sizeof(double) * ((size_t)eb * nb + nb));
        residual_kernel<<<dim3(eb, nb), 256, 0, ctx->stream>>>(AX, X, dtheta, R, ld, g.N, partial);
        DFT_LAUNCH_CHECK();
        rows_sum_kernel2<<<1, 256, 0, ctx->stream>>>(nb, eb, partial, partial + (size_t)eb * nb);
        DFT_LAUNCH_CHECK();
        count_launch(ctx, 2);
        double* hs = pinned(ctx, nb);
        DFT_CUDA(cudaMemcpyAsync(hs, partial + (size_t)eb * nb, sizeof(double) * nb, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        sync(ctx);
        bool occ_conv = true;
        active.clear();
        for (int b = 0; b < nb; ++b) {
            rn[b] = std::isfinite(hs[b]) ? std::sqrt(hs[b] * g.dV) : INFINITY;
            if (!std::isfinite(rn[b])) fail(DFT_NUMERICAL, "non-finite residual in band %d", b);
            // buffer bands only need to stay ahead of the occupied ones
            const double tb = b < nocc ? o.tol : std::max(o.tol, 1e-3);
            if (b < nocc && !(rn[b] < o.tol)) occ_conv = false;
            if (!(rn[b] < tb)) active.push_back(b);
        }
        if (o.verbose) {
            double mx = 0.0;
            for (int b = 0; b < nocc; ++b) mx = std::max(mx, rn[b]);
            fprintf(stderr, "[davidson] it=%d k=%d active=%zu max_occ_res=%.3e theta0=%.10f\n", it, k, active.size(), mx,
                    theta[0]);
        }
        if (tc_mode) {
            double mx = 0.0;
            for (int b = 0; b < nocc; ++b) mx = std::max(mx, rn[b]);
            // also leave the tensor cores when the residuals stop falling: the TF32 hi+lo
            // products have a noise floor that grows with |theta| and the band count
            if (mx < 0.8 * tc_best) {
                tc_best = mx;
                tc_best_it = it;
            }
            const bool stalled = it - tc_best_it >= 15;
            if (occ_conv || mx < o.mixed_switch || stalled) {
                // switch to FP64: restart from the Ritz block, re-orthonormalised and re-projected
                tc_mode = false;
                DFT_CUDA(cudaMemcpyAsync(Vb, X, vecb * nb, cudaMemcpyDeviceToDevice, ctx->stream));
                k = orthonormalise(ctx, g, Vb, 0, Vb, nb, ld, W);
                if (k < nb) fail(DFT_NUMERICAL, "Ritz block lost rank at the FP64 switch");
                apply_hamiltonian(ctx, g, V, Vb, AV, k, ld);
                G.clear();
                grow_G(0, k);
                continue;
            }
        }
        if (occ_conv) {
            done = true;
            break;
        }
        if (it == o.max_iterations) break;
        // ---- corrections ------------------------------------------------------------------
        const int na = (int)active.size();
        if (k + na > kmax) {  // thick restart to the lowest kr Ritz vectors
            const int keep = std::min(k, std::max(nb, std::min(kr, kmax - na)));
            std::vector<double> Zk;
            if (keep > nb) {
                std::vector<double> Gc = G;
                if (!eigh_lowest(k, Gc, keep, w, Zk)) fail(DFT_NUMERICAL, "projected eigensolve failed");
            } else {
                Zk = Z;
            }
            rot(Vb, k, Zk, keep, W);
            DFT_CUDA(cudaMemcpyAsync(Vb, W, vecb * keep, cudaMemcpyDeviceToDevice, ctx->stream));
            rot(AV, k, Zk, keep, W);
            DFT_CUDA(cudaMemcpyAsync(AV, W, vecb * keep, cudaMemcpyDeviceToDevice, ctx->stream));
            k = keep;
            G.assign((size_t)k * k, 0.0);
            for (int i = 0; i < k; ++i) G[(size_t)i * k + i] = w[i];
        }
        if (o.harvest) o.harvest(o.harvest_user, R, ld, active.data(), na, theta.data());
        double* T = Vb + (long long)k * ld;
        DFT_CUDA(cudaMemcpyAsync(dsrc, active.data(), sizeof(int) * na, cudaMemcpyHostToDevice, ctx->stream));
        // auto (-2): one multigrid cycle from 32^3 points on (H2 48^3: 50 eigensolver iterations
        // per SCF instead of 105 with 4 smoothing steps, 35 instead of 44 ms); 4 smoothing
        // steps on smaller grids, whose coarse levels are too few to pay
        const int pc = o.precond_steps == -2 ? (g.N >= 32LL * 32 * 32 ? -1 : 4) : o.precond_steps;
        if (pc == 0) {
            precond_kernel<<<dim3(eb, na), 256, 0, ctx->stream>>>(R, V, dsrc, dtheta, T, ld, g.N, kin);
            DFT_LAUNCH_CHECK();
            count_launch(ctx);
        } else if (pc < 0) {
            // one multigrid cycle for (T + sigma_b) t = r_b, sigma_b = max(-theta_b, 1 Ha)
            precondition_multigrid(ctx, g, R, dsrc, na, dtheta, T, ld);
            // -3: plus the learned correction toward the equation's solution
            if (pc == -3) pnet_precondition(ctx, o.precond_net, g, R, ld, active.data(), na, T);
        } else {
            // (T + sigma_b) t = r_b with sigma_b = max(-theta_b, 1 Ha): the far-field (V ~ 0) form of
            // (H - theta_b) for bound states; t0 = r/d, then damped-Jacobi steps (w = 2/3)
            std::vector<double> sig(na);
            for (int a = 0; a < na; ++a) sig[a] = std::max(-theta[active[a]], 1.0);
            DFT_CUDA(cudaMemcpyAsync(dsigma, sig.data(), sizeof(double) * na, cudaMemcpyHostToDevice, ctx->stream));
            int zc = 32;
            const int sbx = (g.nx + 31) / 32, sby = (g.ny + 7) / 8;
            while (zc > 4 && (long long)sbx * sby * na * ((g.nz + zc - 1) / zc) < 4LL * ctx->num_sms) zc >>= 1;
            const int nzc = (g.nz + zc - 1) / zc;
            if ((long long)na * nzc > 65535) zc = (int)((g.nz + 65535 / na - 1) / (65535 / na)), zc = std::max(zc, 1);
            const int nzc2 = (g.nz + zc - 1) / zc;
            dim3 sgrid(sbx, sby, na * nzc2), sblock(32, 8);
            kinetic_smooth_kernel<<<sgrid, sblock, 0, ctx->stream>>>(g, nullptr, R, dsrc, dsigma, T, ld, zc, nzc2, 1.0);
            double *cur = T, *nxt = W;
            for (int s = 0; s < pc; ++s) {
                kinetic_smooth_kernel<<<sgrid, sblock, 0, ctx->stream>>>(g, cur, R, dsrc, dsigma, nxt, ld, zc, nzc2,
                                                                         2.0 / 3.0);
                std::swap(cur, nxt);
            }
            DFT_LAUNCH_CHECK();
            count_launch(ctx, 1 + pc);
            if (cur != T)
                DFT_CUDA(cudaMemcpyAsync(T, cur, vecb * na, cudaMemcpyDeviceToDevice, ctx->stream));
        }
        int nt = orthonormalise(ctx, g, Vb, k, T, na, ld, W, tc_mode);
        if (nt == 0) {
            // preconditioned directions fell into the basis: fall back to raw residuals
            for (int a = 0; a < na; ++a)
                DFT_CUDA(cudaMemcpyAsync(T + (long long)a * ld, R + (long long)active[a] * ld, vecb,
                                         cudaMemcpyDeviceToDevice, ctx->stream));
            nt = orthonormalise(ctx, g, Vb, k, T, na, ld, W, tc_mode);
            if (nt == 0) fail(DFT_NOT_CONVERGED, "La direccion de expansion Davidson es numericamente dependiente.");
        }
        apply_hamiltonian(ctx, g, V, T, AV + (long long)k * ld, nt, ld);
        grow_G(k, k + nt);
        k += nt;
    }
    // ---- outputs -----------------------------------------------------------------------
    DFT_CUDA(cudaMemcpy2DAsync(psi, vecb, X, vecb, sizeof(double) * (size_t)g.N, nb, cudaMemcpyDeviceToDevice,
                               ctx->stream));
    for (int b = 0; b < nb; ++b) {
        eig_host[b] = theta[b];
        if (resid_host) resid_host[b] = rn[b];
    }
    sync(ctx);
    check_device_status(ctx, "eigensolver");
    if (!done) {
        double mx = 0.0;
        for (int b = 0; b < nocc; ++b) mx = std::max(mx, rn[b]);
        fail(DFT_NOT_CONVERGED, "El orbital molecular no convergio. residual = %g after %d iterations", mx,
             o.max_iterations);
    }
    return it;
}

}  // namespace dftb
