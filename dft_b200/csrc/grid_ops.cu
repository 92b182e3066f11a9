// Grid operators of the 3D Kohn–Sham path on sm_100a: H psi, Jacobi Poisson, XC, density,
// energies, the nuclear potential and the deterministic reductions they need.
//
// Layout: one FP64 array per field, x fastest ((k*ny + j)*nx + i), bands band-major.
// Stencil kernels walk z inside a thread (a "2.5D" march): each thread keeps psi(k-1),
// psi(k), psi(k+1) of its (i,j) column in registers, the x/y neighbours come through L1
// from the lines its warp and block neighbours load, so DRAM sees each value once.
// Every operator whose reference result is deterministic (H psi, Jacobi, density, the
// nuclear potential, mixing) uses round-to-nearest intrinsics in the reference's operation
// order (no FMA contraction), which makes it bit-identical to the reference.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "ops.h"
#include "xc_device.cuh"
#include "xc_grad.cuh"

namespace dftb {

// =============================================================== reductions ==========
namespace {

constexpr int RED_THREADS = 256;

inline int red_blocks(dft_context* ctx, long long n) {
    long long b = (n + RED_THREADS - 1) / RED_THREADS;
    long long cap = (long long)ctx->num_sms * 4;
    return (int)std::max<long long>(1, std::min(b, cap));
}

// K independent sums over p in [0,n): partial[k*gridDim + block]
template <int K, class F>
__global__ void __launch_bounds__(RED_THREADS) reduce_partial_kernel(long long n, F f, double* partial) {
    __shared__ double sh[RED_THREADS / 32];
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        f(p, acc);
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = block_sum(acc[k], sh);
        if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = s;
    }
}

template <int K>
__global__ void reduce_final_kernel(int nblocks, const double* partial, double* out) {
    __shared__ double sh[32];
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partial[k * nblocks + b];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) out[k] = s;
    }
}

}  // namespace

// Runs a K-output reduction and returns the sums on the host (synchronises).
template <int K, class F>
static void reduce_to_host(dft_context* ctx, long long n, F f, double* out_host) {
    const int nb = red_blocks(ctx, n);
    double* partial = (double*)ws_get(ctx, WS_REDUCE, sizeof(double) * ((size_t)K * nb + K));
    double* res = partial + (size_t)K * nb;
    reduce_partial_kernel<K><<<nb, RED_THREADS, 0, ctx->stream>>>(n, f, partial);
    DFT_LAUNCH_CHECK();
    reduce_final_kernel<K><<<1, 256, 0, ctx->stream>>>(nb, partial, res);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    double* h = pinned(ctx, K);
    DFT_CUDA(cudaMemcpyAsync(h, res, sizeof(double) * K, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    for (int k = 0; k < K; ++k) out_host[k] = h[k];
}

struct DotF {
    const double *a, *b;
    __device__ void operator()(long long p, double* acc) const { acc[0] += a[p] * b[p]; }
};
struct Dot3F {
    const double *a, *b;
    double c;
    __device__ void operator()(long long p, double* acc) const { acc[0] += __dmul_rn(__dmul_rn(a[p], b[p]), c); }
};
struct DiffF {
    const double *o, *n;
    __device__ void operator()(long long p, double* acc) const {
        const double d = n[p] - o[p];
        acc[0] += d * d;
        acc[1] += n[p] * n[p];
    }
};

double dot(dft_context* ctx, long long n, const double* a, const double* b) {
    double r;
    reduce_to_host<1>(ctx, n, DotF{a, b}, &r);
    return r;
}

double dot3(dft_context* ctx, long long n, const double* a, const double* b, double c) {
    double r;
    reduce_to_host<1>(ctx, n, Dot3F{a, b, c}, &r);
    return r;
}

// calculateMolecularDensityDifference, reference MolecularSCFHelpers.cpp:46-95
double density_difference(dft_context* ctx, const Grid& g, const double* old_d, const double* new_d) {
    double s[2];
    reduce_to_host<2>(ctx, g.N, DiffF{old_d, new_d}, s);
    const double dn = std::sqrt(s[0] * g.dV), nn = std::sqrt(s[1] * g.dV);
    if (nn <= 1.0e-14) return dn;
    return dn / nn;
}

// =============================================================== elementwise =========
namespace {
__global__ void add2_kernel(long long n, const double* a, const double* b, double* o) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        o[p] = __dadd_rn(a[p], b[p]);
}
__global__ void add3_kernel(long long n, const double* a, const double* b, const double* c, double* o) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        o[p] = __dadd_rn(__dadd_rn(a[p], b[p]), c[p]);
}
__global__ void mix_kernel(long long n, double* d, const double* o, double m) {
    const double om = 1.0 - m;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        d[p] = __dadd_rn(__dmul_rn(om, d[p]), __dmul_rn(m, o[p]));
}
inline int ew_blocks(dft_context* ctx, long long n) {
    long long b = (n + 255) / 256;
    return (int)std::max<long long>(1, std::min<long long>(b, (long long)ctx->num_sms * 8));
}
}  // namespace

void add2(dft_context* ctx, long long n, const double* a, const double* b, double* out) {
    add2_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, a, b, out);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}
void add3(dft_context* ctx, long long n, const double* a, const double* b, const double* c, double* out) {
    add3_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, a, b, c, out);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}
void mix(dft_context* ctx, long long n, double* d, const double* o, double m) {
    mix_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, d, o, m);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
    });
    return fn;
}

// =============================================================== H psi ===============
namespace {

constexpr int HB_X = 32, HB_Y = 8;

// One thread per (i,j) column of one band, marching k over a z-chunk (32 registers, 8 blocks
// per SM).  reference KohnShamHamiltonianMolecule.cpp:59-177: lap = k0*c (+ neighbours in the
// order x-, x+, y-, y+, z-, z+), H psi = -0.5*lap + V*c; absent neighbours are skipped.
__global__ void __launch_bounds__(HB_X* HB_Y) hpsi1_kernel(Grid g, const double* __restrict__ V,
                                                          const double* __restrict__ psi, double* __restrict__ out,
                                                          long long ld, int zchunk, int nzc, double k0) {
    const int i = blockIdx.x * HB_X + threadIdx.x;
    const int j = blockIdx.y * HB_Y + threadIdx.y;
    const int band = blockIdx.z / nzc;
    const int kc = blockIdx.z - band * nzc;
    if (i >= g.nx || j >= g.ny) return;
    const double* __restrict__ p = psi + (long long)band * ld;
    double* __restrict__ o = out + (long long)band * ld;
    const long long sxy = (long long)g.nx * g.ny;
    const int kb = kc * zchunk;
    const int ke = min(g.nz, kb + zchunk);
    long long idx = (long long)kb * sxy + (long long)j * g.nx + i;
    double below = kb > 0 ? __ldg(p + idx - sxy) : 0.0;
    double cur = __ldg(p + idx);
    const bool xl = i > 0, xr = i + 1 < g.nx, yl = j > 0, yr = j + 1 < g.ny;
    for (int k = kb; k < ke; ++k, idx += sxy) {
        const bool zr = k + 1 < g.nz;
        const double above = zr ? __ldg(p + idx + sxy) : 0.0;
        double lap = __dmul_rn(k0, cur);
        if (xl) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx - 1), g.ix2));
        if (xr) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx + 1), g.ix2));
        if (yl) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx - g.nx), g.iy2));
        if (yr) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx + g.nx), g.iy2));
        if (k > 0) lap = __dadd_rn(lap, __dmul_rn(below, g.iz2));
        if (zr) lap = __dadd_rn(lap, __dmul_rn(above, g.iz2));
        o[idx] = __dadd_rn(__dmul_rn(-0.5, lap), __dmul_rn(__ldg(V + idx), cur));
        below = cur;
        cur = above;
    }
}

// hpsi1_kernel with the next plane's loads issued one step ahead ("hpsi_variant" = 3): while
// plane k is computed, psi at k + 2 and V at k + 1 are already in flight, so each thread keeps
// two steps of HBM loads outstanding instead of one.  Same operations in the same order.
__global__ void __launch_bounds__(HB_X* HB_Y, 8) hpsi1p_kernel(Grid g, const double* __restrict__ V,
                                                           const double* __restrict__ psi, double* __restrict__ out,
                                                           long long ld, int zchunk, int nzc, double k0) {
    const int i = blockIdx.x * HB_X + threadIdx.x;
    const int j = blockIdx.y * HB_Y + threadIdx.y;
    const int band = blockIdx.z / nzc;
    const int kc = blockIdx.z - band * nzc;
    if (i >= g.nx || j >= g.ny) return;
    const double* __restrict__ p = psi + (long long)band * ld;
    double* __restrict__ o = out + (long long)band * ld;
    const long long sxy = (long long)g.nx * g.ny;
    const int kb = kc * zchunk;
    const int ke = min(g.nz, kb + zchunk);
    long long idx = (long long)kb * sxy + (long long)j * g.nx + i;
    double below = kb > 0 ? __ldg(p + idx - sxy) : 0.0;
    double cur = __ldg(p + idx);
    double above = kb + 1 < g.nz ? __ldg(p + idx + sxy) : 0.0;
    double v = __ldg(V + idx);
    const bool xl = i > 0, xr = i + 1 < g.nx, yl = j > 0, yr = j + 1 < g.ny;
    for (int k = kb; k < ke; ++k, idx += sxy) {
        const bool zr = k + 1 < g.nz;
        const bool more = k + 1 < ke;  // the next step exists: prefetch its loads
        const double above2 = (more && k + 2 < g.nz) ? __ldg(p + idx + 2 * sxy) : 0.0;
        const double vnext = more ? __ldg(V + idx + sxy) : 0.0;
        double lap = __dmul_rn(k0, cur);
        if (xl) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx - 1), g.ix2));
        if (xr) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx + 1), g.ix2));
        if (yl) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx - g.nx), g.iy2));
        if (yr) lap = __dadd_rn(lap, __dmul_rn(__ldg(p + idx + g.nx), g.iy2));
        if (k > 0) lap = __dadd_rn(lap, __dmul_rn(below, g.iz2));
        if (zr) lap = __dadd_rn(lap, __dmul_rn(above, g.iz2));
        o[idx] = __dadd_rn(__dmul_rn(-0.5, lap), __dmul_rn(v, cur));
        below = cur;
        cur = above;
        above = above2;
        v = vnext;
    }
}

// One thread per (i,j) column of NB bands, marching k over a z-chunk: V is read once per point
// for all NB bands and the NB bands' loads are independent, so more of them are in flight.
// reference KohnShamHamiltonianMolecule.cpp:59-177: lap = k0*c (+ neighbours in the order
// x-, x+, y-, y+, z-, z+), H psi = -0.5*lap + V*c; absent neighbours are skipped.  The
// operation order per band is the reference's, so every band is bit-identical for any NB.
template <int NB>
__global__ void __launch_bounds__(HB_X* HB_Y) hpsi_kernel(Grid g, const double* __restrict__ V,
                                                         const double* __restrict__ psi, double* __restrict__ out,
                                                         long long ld, int nbands, int zchunk, int nzc, double k0) {
    const int i = blockIdx.x * HB_X + threadIdx.x;
    const int j = blockIdx.y * HB_Y + threadIdx.y;
    const int group = blockIdx.z / nzc;
    const int kc = blockIdx.z - group * nzc;
    if (i >= g.nx || j >= g.ny) return;
    const int b0 = group * NB;
    const int nb = min(NB, nbands - b0);
    const double* __restrict__ p = psi + (long long)b0 * ld;
    double* __restrict__ o = out + (long long)b0 * ld;
    const long long sxy = (long long)g.nx * g.ny;
    const int kb = kc * zchunk;
    const int ke = min(g.nz, kb + zchunk);
    long long idx = (long long)kb * sxy + (long long)j * g.nx + i;
    double below[NB], cur[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        below[b] = (b < nb && kb > 0) ? __ldg(p + b * ld + idx - sxy) : 0.0;
        cur[b] = b < nb ? __ldg(p + b * ld + idx) : 0.0;
    }
    const bool xl = i > 0, xr = i + 1 < g.nx, yl = j > 0, yr = j + 1 < g.ny;
    for (int k = kb; k < ke; ++k, idx += sxy) {
        const bool zr = k + 1 < g.nz;
        const double v = __ldg(V + idx);
        double above[NB], xm[NB], xp[NB], ym[NB], yp[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const double* q = p + b * ld + idx;
            const bool on = b < nb;
            above[b] = (on && zr) ? __ldg(q + sxy) : 0.0;
            xm[b] = (on && xl) ? __ldg(q - 1) : 0.0;
            xp[b] = (on && xr) ? __ldg(q + 1) : 0.0;
            ym[b] = (on && yl) ? __ldg(q - g.nx) : 0.0;
            yp[b] = (on && yr) ? __ldg(q + g.nx) : 0.0;
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if (b >= nb) break;
            double lap = __dmul_rn(k0, cur[b]);
            if (xl) lap = __dadd_rn(lap, __dmul_rn(xm[b], g.ix2));
            if (xr) lap = __dadd_rn(lap, __dmul_rn(xp[b], g.ix2));
            if (yl) lap = __dadd_rn(lap, __dmul_rn(ym[b], g.iy2));
            if (yr) lap = __dadd_rn(lap, __dmul_rn(yp[b], g.iy2));
            if (k > 0) lap = __dadd_rn(lap, __dmul_rn(below[b], g.iz2));
            if (zr) lap = __dadd_rn(lap, __dmul_rn(above[b], g.iz2));
            o[b * ld + idx] = __dadd_rn(__dmul_rn(-0.5, lap), __dmul_rn(v, cur[b]));
            below[b] = cur[b];
            cur[b] = above[b];
        }
    }
}

// Tiled variant ("hpsi_variant" = 1): the current plane of a 32 x 8 column tile and its one-point
// halo sit in shared memory, the z neighbours in registers; each thread's load of the next
// plane is issued a full step before it is used.  Same operation order as hpsi_kernel.
template <int NB>
__global__ void __launch_bounds__(HB_X* HB_Y, 6) hpsi_tile_kernel(Grid g, const double* __restrict__ V,
                                                              const double* __restrict__ psi, double* __restrict__ out,
                                                              long long ld, int nbands, int zchunk, int nzc,
                                                              double k0) {
    __shared__ double tile[NB][HB_Y + 2][HB_X + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = blockIdx.x * HB_X + tx;
    const int j = blockIdx.y * HB_Y + ty;
    const int group = blockIdx.z / nzc;
    const int kc = blockIdx.z - group * nzc;
    const int b0 = group * NB;
    const int nb = min(NB, nbands - b0);
    const bool in = i < g.nx && j < g.ny;
    const double* __restrict__ p = psi + (long long)b0 * ld;
    double* __restrict__ o = out + (long long)b0 * ld;
    const long long sxy = (long long)g.nx * g.ny;
    const int kb = kc * zchunk;
    const int ke = min(g.nz, kb + zchunk);
    const long long col = (long long)j * g.nx + i;
    long long idx = (long long)kb * sxy + col;
    // halo duty: x- by tx == 0, x+ by the last column of the tile inside the grid, y- by ty == 0,
    // y+ by the last row inside the grid
    const int last_x = min(HB_X, g.nx - blockIdx.x * HB_X) - 1, last_y = min(HB_Y, g.ny - blockIdx.y * HB_Y) - 1;
    const bool hxm = in && tx == 0 && i > 0, hxp = in && tx == last_x && i + 1 < g.nx;
    const bool hym = in && ty == 0 && j > 0, hyp = in && ty == last_y && j + 1 < g.ny;
    double below[NB], cur[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const bool on = in && b < nb;
        below[b] = (on && kb > 0) ? __ldg(p + b * ld + idx - sxy) : 0.0;
        cur[b] = on ? __ldg(p + b * ld + idx) : 0.0;
    }
    const bool xl = i > 0, xr = i + 1 < g.nx, yl = j > 0, yr = j + 1 < g.ny;
    for (int k = kb; k < ke; ++k, idx += sxy) {
        const bool zr = k + 1 < g.nz;
        double above[NB], hv[NB][4];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const bool on = in && b < nb;
            const double* q = p + b * ld + idx;
            above[b] = (on && zr) ? __ldg(q + sxy) : 0.0;
            hv[b][0] = (on && hxm) ? __ldg(q - 1) : 0.0;
            hv[b][1] = (on && hxp) ? __ldg(q + 1) : 0.0;
            hv[b][2] = (on && hym) ? __ldg(q - g.nx) : 0.0;
            hv[b][3] = (on && hyp) ? __ldg(q + g.nx) : 0.0;
        }
        const double v = in ? __ldg(V + idx) : 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            tile[b][ty + 1][tx + 1] = cur[b];
            if (hxm) tile[b][ty + 1][0] = hv[b][0];
            if (hxp) tile[b][ty + 1][tx + 2] = hv[b][1];
            if (hym) tile[b][0][tx + 1] = hv[b][2];
            if (hyp) tile[b][ty + 2][tx + 1] = hv[b][3];
        }
        __syncthreads();
        if (in) {
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                if (b >= nb) break;
                double lap = __dmul_rn(k0, cur[b]);
                if (xl) lap = __dadd_rn(lap, __dmul_rn(tile[b][ty + 1][tx], g.ix2));
                if (xr) lap = __dadd_rn(lap, __dmul_rn(tile[b][ty + 1][tx + 2], g.ix2));
                if (yl) lap = __dadd_rn(lap, __dmul_rn(tile[b][ty][tx + 1], g.iy2));
                if (yr) lap = __dadd_rn(lap, __dmul_rn(tile[b][ty + 2][tx + 1], g.iy2));
                if (k > 0) lap = __dadd_rn(lap, __dmul_rn(below[b], g.iz2));
                if (zr) lap = __dadd_rn(lap, __dmul_rn(above[b], g.iz2));
                o[b * ld + idx] = __dadd_rn(__dmul_rn(-0.5, lap), __dmul_rn(v, cur[b]));
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            below[b] = cur[b];
            cur[b] = above[b];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- TMA plane ring ---------
// "hpsi_variant" = 2.  Persistent, warp-specialised: a block of 8 compute warps and 1 copy warp
// takes work items (a 32 x 8 column tile, a z-chunk, a run of bands) in turn.  The copy warp's
// first lane walks the planes kb-1 .. ke of every band of its items and loads each plane tile
// with its one-point halo (x from x0-2 so the copy starts on a 16-byte boundary: 36 x 10
// doubles) by cp.async.bulk.tensor into a ring of HT_S shared-memory stages.  Each stage has a
// "full" mbarrier (the copy's transaction count) and an "empty" one (one arrival per compute
// warp when it is done with the plane), so no block-wide barrier paces the march and up to
// HT_S planes per block are in flight.  Compute warp w owns tile row y0 + w (lane = x); the
// point's own column (below, current) is kept in registers.  Out-of-grid parts of a tile are
// zero-filled by the copy and never used: absent neighbours are skipped exactly as in
// hpsi1_kernel, so every value is bit-identical.  V is read from global memory, once per band
// (from L2 after the first band of the run).  Every wait is bounded; a block that gives up sets
// the context's status word and drains its copies.
constexpr int HT_X = 32, HT_Y = 8, HT_S = 8;
constexpr int HT_PX = HT_X + 4, HT_PY = HT_Y + 2;
constexpr int HT_PLANE = HT_PX * HT_PY;                            // doubles in a plane tile
constexpr int HT_STAGE = (HT_PLANE * 8 + 127) / 128 * 128 / 8;     // stage stride (128-byte aligned)
constexpr int HT_THREADS = (HT_Y + 1) * 32;                        // 8 compute warps + 1 copy warp
constexpr long long HT_SPIN = 1LL << 22;                           // polls before a wait gives up

__device__ __forceinline__ uint32_t ht_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool ht_wait(uint64_t* bar, uint32_t parity, long long limit) {
    const uint32_t a = ht_smem(bar);
    for (long long n = 0; n < limit; ++n) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

struct HtWork {
    int bx, by, nzc, zchunk, nbc;
    long long items;  // bx * by * nzc * band runs
};

struct HtItem {
    int x0, y0, kb, ke, b0, nb;
};

__device__ __forceinline__ HtItem ht_item(const HtWork& w, const Grid& g, int nbands, long long it) {
    const long long tiles = (long long)w.bx * w.by;
    const int t = (int)(it % tiles);
    const long long rest = it / tiles;
    const int kc = (int)(rest % w.nzc);
    const int grp = (int)(rest / w.nzc);
    HtItem r;
    r.x0 = (t % w.bx) * HT_X;
    r.y0 = (t / w.bx) * HT_Y;
    r.kb = kc * w.zchunk;
    r.ke = min(g.nz, r.kb + w.zchunk);
    r.b0 = grp * w.nbc;
    r.nb = min(w.nbc, nbands - r.b0);
    return r;
}

__global__ void __launch_bounds__(HT_THREADS, 4) hpsi_tma_kernel(const __grid_constant__ CUtensorMap tm, Grid g,
                                                                 const double* __restrict__ V, double* __restrict__ out,
                                                                 long long ld, int nbands, HtWork w, double k0,
                                                                 int* __restrict__ status) {
    __shared__ __align__(128) double plane[HT_S][HT_STAGE];
    __shared__ __align__(8) uint64_t full[HT_S];
    __shared__ __align__(8) uint64_t empty[HT_S];
    __shared__ int abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < HT_S; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ht_smem(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(ht_smem(&empty[s])), "r"(HT_Y));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abort_flag = 0;
    }
    __syncthreads();
    volatile int* abort_v = &abort_flag;
    if (warp == HT_Y) {
        // copy warp: its first lane issues every plane of this block's items in order
        if (lane == 0) {
            long long P = 0;
            bool ok = true;
            for (long long it = blockIdx.x; it < w.items && ok; it += gridDim.x) {
                const HtItem m = ht_item(w, g, nbands, it);
                for (int b = 0; b < m.nb && ok; ++b)
                    for (int k = m.kb - 1; k <= m.ke; ++k, ++P) {
                        const int s = (int)(P % HT_S);
                        // stage s is free once every compute warp released plane P - HT_S
                        if (!ht_wait(&empty[s], (uint32_t)(((P / HT_S) & 1) ^ 1), HT_SPIN) || *abort_v) {
                            ok = false;
                            break;
                        }
                        const uint32_t bar = ht_smem(&full[s]);
                        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                                     "r"(HT_PLANE * 8)
                                     : "memory");
                        asm volatile(
                            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], "
                            "[%1, {%2, %3, %4, %5}], [%6];" ::"r"(ht_smem(&plane[s][0])),
                            "l"(reinterpret_cast<uint64_t>(&tm)), "r"(m.x0 - 2), "r"(m.y0 - 1), "r"(k),
                            "r"(m.b0 + b), "r"(bar)
                            : "memory");
                    }
            }
            if (!ok) {
                *abort_v = 1;
                atomicOr(status, 1);
            }
            // the copies of the last HT_S planes may still be in flight: let them land
            for (long long q = P > HT_S ? P - HT_S : 0; q < P; ++q)
                ht_wait(&full[q % HT_S], (uint32_t)((q / HT_S) & 1), HT_SPIN);
        }
    } else {
        // compute warp: tile row y0 + warp, point x0 + lane
        const int c = (warp + 1) * HT_PX + lane + 2;  // the point's offset inside a plane tile
        const long long sxy = (long long)g.nx * g.ny;
        long long P = 0;
        bool ok = true;
        auto release = [&](long long q) {
            __syncwarp();
            if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(ht_smem(&empty[q % HT_S])) : "memory");
        };
        for (long long it = blockIdx.x; it < w.items && ok; it += gridDim.x) {
            const HtItem m = ht_item(w, g, nbands, it);
            const int i = m.x0 + lane, j = m.y0 + warp;
            const bool in = i < g.nx && j < g.ny;
            const bool xl = i > 0, xr = i + 1 < g.nx, yl = j > 0, yr = j + 1 < g.ny;
            const int nk = m.ke - m.kb;
            for (int b = 0; b < m.nb && ok; ++b) {
                // planes P (kb - 1), P + 1 (kb), ..., P + nk + 1 (ke) of this band
                if (!ht_wait(&full[P % HT_S], (uint32_t)((P / HT_S) & 1), HT_SPIN) ||
                    !ht_wait(&full[(P + 1) % HT_S], (uint32_t)(((P + 1) / HT_S) & 1), HT_SPIN)) {
                    ok = false;
                    break;
                }
                double below = plane[P % HT_S][c];
                double cur = plane[(P + 1) % HT_S][c];
                release(P);
                double* __restrict__ o = out + (long long)(m.b0 + b) * ld;
                for (int k = m.kb; k < m.ke; ++k) {
                    const long long q = P + 1 + (k - m.kb);
                    const long long idx = (long long)k * sxy + (long long)j * g.nx + i;
                    const double v = in ? __ldg(V + idx) : 0.0;
                    if (!ht_wait(&full[(q + 1) % HT_S], (uint32_t)(((q + 1) / HT_S) & 1), HT_SPIN)) {
                        ok = false;
                        break;
                    }
                    const double* Pl = plane[q % HT_S];
                    const double above = plane[(q + 1) % HT_S][c];
                    if (in) {
                        double lap = __dmul_rn(k0, cur);
                        if (xl) lap = __dadd_rn(lap, __dmul_rn(Pl[c - 1], g.ix2));
                        if (xr) lap = __dadd_rn(lap, __dmul_rn(Pl[c + 1], g.ix2));
                        if (yl) lap = __dadd_rn(lap, __dmul_rn(Pl[c - HT_PX], g.iy2));
                        if (yr) lap = __dadd_rn(lap, __dmul_rn(Pl[c + HT_PX], g.iy2));
                        if (k > 0) lap = __dadd_rn(lap, __dmul_rn(below, g.iz2));
                        if (k + 1 < g.nz) lap = __dadd_rn(lap, __dmul_rn(above, g.iz2));
                        o[idx] = __dadd_rn(__dmul_rn(-0.5, lap), __dmul_rn(v, cur));
                    }
                    release(q);
                    below = cur;
                    cur = above;
                }
                if (!ok) break;
                release(P + nk + 1);  // plane ke
                P += nk + 2;
            }
        }
        if (!ok) *abort_v = 1;
    }
    __syncthreads();
}

}  // namespace

// The TMA ring needs 16-byte strides (nx and ld even) and a 16-byte aligned band block.
bool hpsi_tma_eligible(const Grid& g, const double* psi, long long ld) {
    return g.nx % 2 == 0 && ld % 2 == 0 && (reinterpret_cast<uintptr_t>(psi) & 15) == 0 && g.nx >= 3 &&
           g.ny >= 3 && tensor_map_encoder() != nullptr;
}

namespace {

// 4-D map (x, y, z, band) of nbands bands at psi, box = one plane tile with its halo.
CUtensorMap hpsi_tensor_map(const Grid& g, const double* psi, long long ld, int nbands) {
    CUtensorMap tm;
    const cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)nbands};
    const cuuint64_t strides[3] = {(cuuint64_t)g.nx * 8, (cuuint64_t)g.nx * g.ny * 8, (cuuint64_t)ld * 8};
    const cuuint32_t box[4] = {HT_PX, HT_PY, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = tensor_map_encoder()(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(psi), dims,
                                            strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(DFT_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return tm;
}

inline int pick_zchunk(const Grid& g, long long columns_blocks, int nbands, int num_sms) {
    // enough CTAs to fill the machine a few times over, but chunks long enough to amortise
    // the two-plane warm-up of the z march
    int zc = 32;
    while (zc > 4 && columns_blocks * nbands * ((g.nz + zc - 1) / zc) < 4LL * num_sms) zc >>= 1;
    return zc;
}

}  // namespace

int* device_status(dft_context* ctx) {
    if (!ctx->dev_status) {
        DFT_CUDA(cudaMalloc(&ctx->dev_status, 256));
        DFT_CUDA(cudaMemsetAsync(ctx->dev_status, 0, 256, ctx->stream));
    }
    return ctx->dev_status;
}

void check_device_status(dft_context* ctx, const char* what) {
    if (!ctx->dev_status) return;
    int* h = (int*)pinned(ctx, 1);
    DFT_CUDA(cudaMemcpyAsync(h, ctx->dev_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    if (*h) {
        DFT_CUDA(cudaMemsetAsync(ctx->dev_status, 0, sizeof(int), ctx->stream));
        fail(DFT_CUDA_ERROR, "%s: a bounded device wait gave up (status %d)", what, *h);
    }
}

void apply_hamiltonian(dft_context* ctx, const Grid& g, const double* V, const double* psi, double* hpsi, int nbands,
                       long long ld) {
    if (nbands <= 0) return;
    const double k0 = -2.0 * (g.ix2 + g.iy2 + g.iz2);
    // variant: the "hpsi_variant" key, else the autotuner's choice for this grid
    int variant = ctx->hpsi_variant;
    const auto tuned = ctx->tuned.find({(long long)g.nx, (long long)g.ny, (long long)g.nz});
    if (variant == 0 && tuned != ctx->tuned.end()) variant = tuned->second[2];
    if (variant == 2 && hpsi_tma_eligible(g, psi, ld)) {
        // bands per item: the "hpsi_bands_per_thread" key (1, 2, 4 or 8), else the tuned value, else 4
        int nbc = ctx->hpsi_bands_per_thread > 0 ? ctx->hpsi_bands_per_thread
                  : tuned != ctx->tuned.end() && tuned->second[2] == 2 ? tuned->second[0] : 4;
        nbc = std::max(1, std::min(nbc, nbands));
        static int per_sm = 0;
        if (!per_sm) {
            DFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hpsi_tma_kernel, HT_THREADS, 0));
            per_sm = std::max(per_sm, 1);
        }
        const long long slots = (long long)per_sm * ctx->num_sms;
        HtWork w{};
        w.bx = (g.nx + HT_X - 1) / HT_X;
        w.by = (g.ny + HT_Y - 1) / HT_Y;
        w.nbc = nbc;
        const long long runs = (nbands + nbc - 1) / nbc;
        // z-chunks long enough to amortise the two extra planes, short enough for ~3 items per block
        w.zchunk = 64;
        while (w.zchunk > 8 && (long long)w.bx * w.by * runs * ((g.nz + w.zchunk - 1) / w.zchunk) < 3 * slots)
            w.zchunk >>= 1;
        w.nzc = (g.nz + w.zchunk - 1) / w.zchunk;
        w.items = (long long)w.bx * w.by * w.nzc * runs;
        const int grid = (int)std::min<long long>(w.items, slots);
        const CUtensorMap tm = hpsi_tensor_map(g, psi, ld, nbands);
        hpsi_tma_kernel<<<grid, HT_THREADS, 0, ctx->stream>>>(tm, g, V, hpsi, ld, nbands, w, k0, device_status(ctx));
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        return;
    }
    dim3 block(HB_X, HB_Y);
    const int bx = (g.nx + HB_X - 1) / HB_X, by = (g.ny + HB_Y - 1) / HB_Y;
    // bands per thread: the "hpsi_bands_per_thread" tuning key, else the autotuner's choice for
    // this grid, else 1 (the 32-register single-band march keeps 8 blocks per SM resident)
    int nbt = ctx->hpsi_bands_per_thread;
    if (nbt <= 0) {
        auto t = ctx->tuned.find({(long long)g.nx, (long long)g.ny, (long long)g.nz});
        nbt = t != ctx->tuned.end() ? t->second[0] : 1;
    }
    nbt = std::min(nbt, std::max(1, nbands));
    nbt = nbt >= 4 ? 4 : nbt >= 2 ? 2 : 1;
    if (ctx->hpsi_variant == 1) nbt = std::min(nbt, 2);
    if (variant == 3) nbt = 1;  // the prefetching march is single-band
    const int groups = (nbands + nbt - 1) / nbt;
    // z-chunk: the "hpsi_zchunk" key (points per block's march), else enough blocks to fill the
    // machine a few times over
    int zset = ctx->hpsi_zchunk;
    if (zset == 0 && tuned != ctx->tuned.end()) zset = tuned->second[3];
    const int zc = zset > 0 ? std::min(zset, g.nz) : pick_zchunk(g, (long long)bx * by, groups, ctx->num_sms);
    const int nzc = (g.nz + zc - 1) / zc;
    // gridDim.z limit is 65535: split the band block if needed
    const int max_groups = std::max(1, 65535 / nzc);
    for (int g0 = 0; g0 < groups; g0 += max_groups) {
        const int ng = std::min(max_groups, groups - g0);
        const int b0 = g0 * nbt;
        const int nb = std::min(nbands - b0, ng * nbt);
        dim3 grid(bx, by, ng * nzc);
        const double* pi = psi + (long long)b0 * ld;
        double* po = hpsi + (long long)b0 * ld;
        if (ctx->hpsi_variant == 1) {
            if (nbt >= 2) hpsi_tile_kernel<2><<<grid, block, 0, ctx->stream>>>(g, V, pi, po, ld, nb, zc, nzc, k0);
            else hpsi_tile_kernel<1><<<grid, block, 0, ctx->stream>>>(g, V, pi, po, ld, nb, zc, nzc, k0);
        } else if (nbt == 4) {
            hpsi_kernel<4><<<grid, block, 0, ctx->stream>>>(g, V, pi, po, ld, nb, zc, nzc, k0);
        } else if (nbt == 2) {
            hpsi_kernel<2><<<grid, block, 0, ctx->stream>>>(g, V, pi, po, ld, nb, zc, nzc, k0);
        } else if (variant == 3) {
            hpsi1p_kernel<<<grid, block, 0, ctx->stream>>>(g, V, pi, po, ld, zc, nzc, k0);
        } else {
            hpsi1_kernel<<<grid, block, 0, ctx->stream>>>(g, V, pi, po, ld, zc, nzc, k0);
        }
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
}

// =============================================================== Jacobi Poisson ======
namespace {

struct JacobiCtrl {
    unsigned long long diff_bits;  // running max |dV| of the sweep in flight (as uint64 of a non-negative double)
    unsigned int ticket;           // blocks finished in the sweep in flight
    int done;                      // 1 once the stop rule fired or the cap was reached
    long long sweep;               // completed sweeps; the current iterate lives in buf[sweep & 1]
    double last_diff;              // max |dV| of the last completed sweep
};

// Boundary fill, reference HartreePotentialMolecule.cpp:37-95 and :171-202.  Interior = 0
// (the reference's cold start, :152-155) or, for a warm start, the interior of `guess`
// (which may alias `a`).  x_i = xmin + i*dx exactly as CartesianGrid::getX; Q is the total charge.
__global__ void jacobi_init_kernel(Grid g, double Q, double* a, double* b, const double* guess) {
    const long long n = g.N;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx);
        const int j = (int)((p / g.nx) % g.ny);
        const int k = (int)(p / ((long long)g.nx * g.ny));
        double v = 0.0;
        const bool face = i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz;
        if (!face && guess) v = guess[p];
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
                if (r > 0.0) v = Q / r;
            }
        }
        a[p] = v;
        b[p] = v;
    }
}

// Sequential total charge (the reference's summation order), used only when a boundary
// face is not exactly on a node so boundary values are non-zero.
__global__ void total_charge_seq_kernel(long long n, const double* rho, double dV, double* out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double s = 0.0;
        for (long long p = 0; p < n; ++p) s += rho[p];
        *out = s * dV;
    }
}

constexpr int JB_X = 32, JB_Y = 8;

// One Jacobi sweep over the interior (reference HartreePotentialMolecule.cpp:207-321):
// V' = (ix2 (V[x-]+V[x+]) + iy2 (V[y-]+V[y+]) + iz2 (V[z-]+V[z+]) + 4 pi rho) / den,
// max |V'-V| folded into ctrl; the last block to finish closes the sweep.
__global__ void __launch_bounds__(JB_X* JB_Y) jacobi_sweep_kernel(Grid g, const double* __restrict__ rho,
                                                                  double* buf0, double* buf1, JacobiCtrl* ctrl,
                                                                  double den, double tol, long long cap,
                                                                  int zchunk) {
    __shared__ double sh[JB_X * JB_Y / 32];
    __shared__ int s_done;
    __shared__ long long s_sweep;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        s_done = __ldcg(&ctrl->done);
        s_sweep = __ldcg(&ctrl->sweep);
    }
    __syncthreads();
    if (s_done) return;
    const double* __restrict__ cur = (s_sweep & 1) ? buf1 : buf0;
    double* __restrict__ nxt = (s_sweep & 1) ? buf0 : buf1;
    const double c4pi = 4.0 * xcf::PI;
    const int i = blockIdx.x * JB_X + threadIdx.x;
    const int j = blockIdx.y * JB_Y + threadIdx.y;
    double md = 0.0;
    if (i >= 1 && i + 1 < g.nx && j >= 1 && j + 1 < g.ny) {
        // 32-bit offsets (the host rejects grids of 2^31 points or more)
        const int sxy = g.nx * g.ny;
        const int kb = max(1, (int)blockIdx.z * zchunk);
        const int ke = min(g.nz - 1, (int)(blockIdx.z + 1) * zchunk);
        if (kb < ke) {
            int idx = kb * sxy + j * g.nx + i;
            double below = __ldg(cur + idx - sxy);
            double c = __ldg(cur + idx);
            // unrolled so that the loads of several planes are in flight together
#pragma unroll 4
            for (int k = kb; k < ke; ++k, idx += sxy) {
                const double above = __ldg(cur + idx + sxy);
                const double sx = __dadd_rn(__ldg(cur + idx - 1), __ldg(cur + idx + 1));
                const double sy = __dadd_rn(__ldg(cur + idx - g.nx), __ldg(cur + idx + g.nx));
                const double sz = __dadd_rn(below, above);
                double acc = __dadd_rn(__dmul_rn(g.ix2, sx), __dmul_rn(g.iy2, sy));
                acc = __dadd_rn(acc, __dmul_rn(g.iz2, sz));
                acc = __dadd_rn(acc, __dmul_rn(c4pi, __ldg(rho + idx)));
                const double v = __ddiv_rn(acc, den);
                nxt[idx] = v;
                md = fmax(md, fabs(v - c));
                below = c;
                c = above;
            }
        }
    }
    // block max -> global max (non-negative doubles order like their bit patterns)
    const int tid = threadIdx.y * JB_X + threadIdx.x;
    md = warp_max(md);
    if ((tid & 31) == 0) sh[tid >> 5] = md;
    __syncthreads();
    if (tid == 0) {
        double m = sh[0];
        for (int w = 1; w < JB_X * JB_Y / 32; ++w) m = fmax(m, sh[w]);
        atomicMax(&ctrl->diff_bits, (unsigned long long)__double_as_longlong(m));
        __threadfence();
        const unsigned int total = gridDim.x * gridDim.y * gridDim.z;
        const unsigned int t = atomicAdd(&ctrl->ticket, 1u);
        if (t == total - 1) {
            __threadfence();
            const double d = __longlong_as_double((long long)atomicExch(&ctrl->diff_bits, 0ull));
            ctrl->ticket = 0;
            ctrl->last_diff = d;
            ctrl->sweep = s_sweep + 1;
            if (d < tol || s_sweep + 1 >= cap) ctrl->done = 1;
            __threadfence();
        }
    }
}

// ---- temporally blocked Jacobi: up to TMAX sweeps per launch -----------------------------
//
// A block owns a (32-2*TMAX)^2 column tile and a z-chunk of the output and holds a 32 x 32
// column region (tile + TMAX halo) in shared memory.  It marches z: each step loads one input
// plane (level 0) and advances every time level t = 1..tsw by one plane (level t computes
// plane zin - t from the three level-(t-1) planes around it, kept in a 3-plane ring per level).
// Each level is exactly one Jacobi sweep of the reference (same arithmetic as
// jacobi_sweep_kernel); halo columns and the z-halo of the chunk are recomputed redundantly
// and discarded.  Per-level max|dV| over owned points goes to ctrl->level_bits[t]; the last
// block to finish finds the first level that met the stop rule (or the cap).  If that level
// is below tsw the host replays the launch from its (untouched) input with fewer levels.
constexpr int TB_R = 32;  // region edge (columns)

struct JacobiTBCtrl {
    unsigned long long level_bits[9];  // running max |dV| per level of the launch in flight
    unsigned int ticket;
    int done;
    long long sweep;        // sweeps completed by finished launches
    long long launches;     // finished launches; the input of launch L is buf[L & 1]
    int final_level;        // level of the launch that met the stop rule
    int final_in_parity;    // input parity of that launch
    double last_diff;
};

template <int TMAX>
__global__ void __launch_bounds__(TB_R* TB_R, 1)
    jacobi_tb_kernel(Grid g, const double* __restrict__ rho, double* buf0, double* buf1, JacobiTBCtrl* ctrl,
                     double den, double tol, long long cap, int zchunk, int tsw, int replay_parity) {
    extern __shared__ double ring[];  // [TMAX levels][3 slots][TB_R][TB_R]
    __shared__ double red[TB_R][TMAX + 1];
    __shared__ int s_done;
    __shared__ long long s_sweep, s_launch;
    const bool replay = replay_parity >= 0;
    const int rx = threadIdx.x, ry = threadIdx.y, tid = ry * TB_R + rx;
    if (tid == 0) {
        if (replay) {
            s_done = 0;
            s_launch = replay_parity;
            s_sweep = 0;
        } else {
            s_done = __ldcg(&ctrl->done);
            s_launch = __ldcg(&ctrl->launches);
            s_sweep = __ldcg(&ctrl->sweep);
        }
    }
    __syncthreads();
    if (s_done) return;
    const double* __restrict__ vin = (s_launch & 1) ? buf1 : buf0;
    double* __restrict__ vout = (s_launch & 1) ? buf0 : buf1;
    constexpr int TT = TB_R - 2 * TMAX;  // owned tile edge
    const int x = (int)blockIdx.x * TT - TMAX + rx;
    const int y = (int)blockIdx.y * TT - TMAX + ry;
    const bool in_grid = x >= 0 && x < g.nx && y >= 0 && y < g.ny;
    const bool edge_col = x == 0 || x == g.nx - 1 || y == 0 || y == g.ny - 1;
    const bool owned = in_grid && rx >= TMAX && rx < TMAX + TT && ry >= TMAX && ry < TMAX + TT;
    const int z0 = (int)blockIdx.z * zchunk;
    const int z1 = min(g.nz, z0 + zchunk);
    const long long sxy = (long long)g.nx * g.ny;
    const long long col = (long long)y * g.nx + x;
    const double c4pi = 4.0 * xcf::PI;
    constexpr int PL = TB_R * TB_R;
    auto cell = [&](int level, int z, int dx, int dy) -> double& {
        return ring[((level * 3 + ((z % 3) + 3) % 3) * PL) + (ry + dy) * TB_R + (rx + dx)];
    };
    double md[TMAX + 1];
    double rr[TMAX + 1];  // rr[t] = rho of this column at plane zin - t (level t's source term)
#pragma unroll
    for (int t = 0; t <= TMAX; ++t) md[t] = rr[t] = 0.0;
    auto load = [&](const double* f, int z) -> double {
        return (in_grid && z >= 0 && z < g.nz) ? __ldg(f + (long long)z * sxy + col) : 0.0;
    };
    // one plane of V and of rho are fetched a step ahead, so their latency overlaps the levels
    double vpre = load(vin, z0 - tsw), rpre = 0.0;
    for (int zin = z0 - tsw; zin < z1 + tsw; ++zin) {
#pragma unroll
        for (int t = TMAX; t >= 2; --t) rr[t] = rr[t - 1];
        rr[1] = rpre;
        if (zin >= 0 && zin < g.nz) cell(0, zin, 0, 0) = vpre;
        vpre = load(vin, zin + 1);
        rpre = load(rho, zin);
        __syncthreads();
#pragma unroll
        for (int t = 1; t <= TMAX; ++t) {
            if (t <= tsw) {
                const int zt = zin - t;
                const bool active = zt >= 0 && zt < g.nz && zt >= z0 - (tsw - t) && zt < z1 + (tsw - t);
                if (active) {
                    const double c = cell(t - 1, zt, 0, 0);
                    double v = c;
                    const bool interior = in_grid && !edge_col && zt > 0 && zt < g.nz - 1 && rx > 0 &&
                                          rx < TB_R - 1 && ry > 0 && ry < TB_R - 1;
                    if (interior) {
                        const double sx = __dadd_rn(cell(t - 1, zt, -1, 0), cell(t - 1, zt, 1, 0));
                        const double sy = __dadd_rn(cell(t - 1, zt, 0, -1), cell(t - 1, zt, 0, 1));
                        const double sz = __dadd_rn(cell(t - 1, zt - 1, 0, 0), cell(t - 1, zt + 1, 0, 0));
                        double acc = __dadd_rn(__dmul_rn(g.ix2, sx), __dmul_rn(g.iy2, sy));
                        acc = __dadd_rn(acc, __dmul_rn(g.iz2, sz));
                        acc = __dadd_rn(acc, __dmul_rn(c4pi, rr[t]));
                        v = __ddiv_rn(acc, den);
                        if (owned && zt >= z0 && zt < z1) md[t] = fmax(md[t], fabs(v - c));
                    }
                    if (t == tsw) {
                        if (owned && zt >= z0 && zt < z1) vout[(long long)zt * sxy + col] = v;
                    } else {
                        cell(t, zt, 0, 0) = v;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (replay) return;
    // per-level block max -> global per-level max
#pragma unroll
    for (int t = 1; t <= TMAX; ++t) {
        double m = warp_max(md[t]);
        if (rx == 0) red[ry][t] = m;
    }
    __syncthreads();
    if (tid == 0) {
        for (int t = 1; t <= tsw; ++t) {
            double m = 0.0;
            for (int w = 0; w < TB_R; ++w) m = fmax(m, red[w][t]);
            atomicMax(&ctrl->level_bits[t], (unsigned long long)__double_as_longlong(m));
        }
        __threadfence();
        const unsigned int total = gridDim.x * gridDim.y * gridDim.z;
        if (atomicAdd(&ctrl->ticket, 1u) == total - 1) {
            __threadfence();
            int fin = 0;
            double dlast = 0.0;
            for (int t = 1; t <= tsw; ++t) {
                const double d = __longlong_as_double((long long)atomicExch(&ctrl->level_bits[t], 0ull));
                if (!fin) {
                    dlast = d;
                    if (d < tol || s_sweep + t >= cap) fin = t;
                }
            }
            ctrl->ticket = 0;
            ctrl->last_diff = dlast;
            if (fin) {
                ctrl->done = 1;
                ctrl->final_level = fin;
                ctrl->final_in_parity = (int)(s_launch & 1);
                ctrl->sweep = s_sweep + fin;
            } else {
                ctrl->sweep = s_sweep + tsw;
            }
            ctrl->launches = s_launch + 1;
            __threadfence();
        }
    }
}

// ---- persistent Jacobi: the whole solve in one cooperative launch --------------------------
// For small grids the sweep is a few microseconds of work and launch latency dominates.  All
// blocks stay resident (cooperative launch) and meet at a grid barrier after every sweep;
// every block reads the same global max|dV| after the barrier, so all stop at the same sweep.
// Loads of the iterates bypass L1 (__ldcg): other SMs rewrite them every sweep.
// The barrier wait is bounded: a block that polls poll_limit times (2^24 unless the
// "grid_barrier_poll_limit" tuning key says otherwise) without seeing the barrier open sets
// ctrl->error and leaves, and so do the others at their next barrier; the host reports it.
struct JacobiPCtrl {
    unsigned long long slot[3];  // per-sweep max |dV| (sweep s uses slot s % 3)
    unsigned int count;          // grid barrier arrivals
    unsigned int gen;            // grid barrier generation
    int error;
    int pad;
    long long sweeps;
    double last_diff;
};

__device__ __forceinline__ bool grid_barrier(JacobiPCtrl* c, unsigned int nblocks, long long poll_limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        int ok = 1;
        const unsigned int gen = atomicAdd(&c->gen, 0u);
        __threadfence();
        if (atomicAdd(&c->count, 1u) == nblocks - 1) {
            atomicExch(&c->count, 0u);
            __threadfence();
            atomicAdd(&c->gen, 1u);
        } else {
            long long polls = 0;
            while (atomicAdd(&c->gen, 0u) == gen) {
                if (++polls >= poll_limit || atomicAdd(&c->error, 0) != 0) {
                    atomicExch(&c->error, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__global__ void __launch_bounds__(256) jacobi_persistent_kernel(Grid g, const double* __restrict__ rho, double* buf0,
                                                                double* buf1, JacobiPCtrl* ctrl, double den, double tol,
                                                                long long cap, long long poll_limit) {
    __shared__ double sh[8];
    __shared__ double s_d;
    const double c4pi = 4.0 * xcf::PI;
    const long long sxy = (long long)g.nx * g.ny;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const unsigned int nblocks = gridDim.x;
    for (long long s = 0; s < cap; ++s) {
        const double* cur = (s & 1) ? buf1 : buf0;
        double* nxt = (s & 1) ? buf0 : buf1;
        double md = 0.0;
        for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += stride) {
            const int i = (int)(p % g.nx);
            const int j = (int)((p / g.nx) % g.ny);
            const int k = (int)(p / sxy);
            if (i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz) continue;
            const double c = __ldcg(cur + p);
            const double sx = __dadd_rn(__ldcg(cur + p - 1), __ldcg(cur + p + 1));
            const double sy = __dadd_rn(__ldcg(cur + p - g.nx), __ldcg(cur + p + g.nx));
            const double sz = __dadd_rn(__ldcg(cur + p - sxy), __ldcg(cur + p + sxy));
            double acc = __dadd_rn(__dmul_rn(g.ix2, sx), __dmul_rn(g.iy2, sy));
            acc = __dadd_rn(acc, __dmul_rn(g.iz2, sz));
            acc = __dadd_rn(acc, __dmul_rn(c4pi, __ldg(rho + p)));
            const double v = __ddiv_rn(acc, den);
            __stcg(nxt + p, v);
            md = fmax(md, fabs(v - c));
        }
        md = warp_max(md);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = md;
        __syncthreads();
        if (threadIdx.x == 0) {
            double m = sh[0];
            for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
            atomicMax(&ctrl->slot[s % 3], (unsigned long long)__double_as_longlong(m));
        }
        if (!grid_barrier(ctrl, nblocks, poll_limit)) return;
        if (threadIdx.x == 0) {
            s_d = __longlong_as_double((long long)atomicAdd(&ctrl->slot[s % 3], 0ull));
            if (blockIdx.x == 0) atomicExch(&ctrl->slot[(s + 2) % 3], 0ull);  // read by all before barrier s
        }
        __syncthreads();
        const double d = s_d;
        if (d < tol || s + 1 >= cap) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                ctrl->sweeps = s + 1;
                ctrl->last_diff = d;
            }
            return;
        }
    }
}

// ---- cluster-resident Jacobi: the whole grid in the shared memory of one thread-block cluster
// Small grids (C1 is 48^3 = 110,592 points, 0.9 MB per field) fit in the distributed shared
// memory of a 16-block cluster: block r keeps a z-slab of V, V' and rho in its own shared memory
// and reads the two halo planes from its neighbours' shared memory (DSMEM).  One hardware
// cluster barrier per sweep; after it every block reads the 16 per-block maxima, so all blocks
// take the same stop decision.  Same arithmetic as jacobi_sweep_kernel (bit-identical).
constexpr int JC_THREADS = 1024;

struct JacobiClusterOut {
    long long sweeps;
    double last_diff;
};

__global__ void __launch_bounds__(JC_THREADS, 1)
    jacobi_cluster_kernel(Grid g, const double* __restrict__ rho, double* __restrict__ vh, JacobiClusterOut* out,
                          double den, double tol, long long cap, int pmax) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int nr = (int)cl.num_blocks();
    const int r = (int)cl.block_rank();
    extern __shared__ double sm[];
    __shared__ double s_max[2];
    __shared__ double red[JC_THREADS / 32];
    __shared__ double s_d;
    const int plane = g.nx * g.ny;
    double* bufA = sm;
    double* bufB = sm + (size_t)pmax * plane;
    double* R = sm + 2 * (size_t)pmax * plane;
    const int zlo = (int)(((long long)r * g.nz) / nr), zhi = (int)(((long long)(r + 1) * g.nz) / nr);
    const int np = zhi - zlo;
    const int zlo_prev = r > 0 ? (int)(((long long)(r - 1) * g.nz) / nr) : 0;
    const int np_prev = zlo - zlo_prev;
    const int tid = threadIdx.x;
    for (int e = tid; e < np * plane; e += JC_THREADS) {
        const double v = vh[(size_t)zlo * plane + e];
        bufA[e] = v;
        bufB[e] = v;
        R[e] = rho[(size_t)zlo * plane + e];
    }
    // neighbour slabs (never dereferenced at the outer faces: planes 0 and nz-1 are fixed)
    double* A_prev = r > 0 ? cl.map_shared_rank(bufA, r - 1) : nullptr;
    double* B_prev = r > 0 ? cl.map_shared_rank(bufB, r - 1) : nullptr;
    double* A_next = r + 1 < nr ? cl.map_shared_rank(bufA, r + 1) : nullptr;
    double* B_next = r + 1 < nr ? cl.map_shared_rank(bufB, r + 1) : nullptr;
    cl.sync();
    const double c4pi = 4.0 * xcf::PI;
    long long fin = 0;
    double d = 0.0;
    for (long long s = 0; s < cap; ++s) {
        const bool odd = s & 1;
        const double* cur = odd ? bufB : bufA;
        double* nxt = odd ? bufA : bufB;
        const double* cprev = odd ? B_prev : A_prev;
        const double* cnext = odd ? B_next : A_next;
        double md = 0.0;
        for (int lp = 0; lp < np; ++lp) {
            const int z = zlo + lp;
            if (z == 0 || z == g.nz - 1) continue;
            const double* zm_plane = lp > 0 ? cur + (size_t)(lp - 1) * plane : cprev + (size_t)(np_prev - 1) * plane;
            const double* zp_plane = lp + 1 < np ? cur + (size_t)(lp + 1) * plane : cnext;
            const double* cp = cur + (size_t)lp * plane;
            double* np_out = nxt + (size_t)lp * plane;
            const double* rp = R + (size_t)lp * plane;
            for (int q = tid; q < plane; q += JC_THREADS) {
                const int j = q / g.nx, i = q - j * g.nx;
                if (i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1) continue;
                const double c = cp[q];
                const double sx = __dadd_rn(cp[q - 1], cp[q + 1]);
                const double sy = __dadd_rn(cp[q - g.nx], cp[q + g.nx]);
                const double sz = __dadd_rn(zm_plane[q], zp_plane[q]);
                double acc = __dadd_rn(__dmul_rn(g.ix2, sx), __dmul_rn(g.iy2, sy));
                acc = __dadd_rn(acc, __dmul_rn(g.iz2, sz));
                acc = __dadd_rn(acc, __dmul_rn(c4pi, rp[q]));
                const double v = __ddiv_rn(acc, den);
                np_out[q] = v;
                md = fmax(md, fabs(v - c));
            }
        }
        md = warp_max(md);
        if ((tid & 31) == 0) red[tid >> 5] = md;
        __syncthreads();
        if (tid == 0) {
            double m = red[0];
            for (int w = 1; w < JC_THREADS / 32; ++w) m = fmax(m, red[w]);
            s_max[s & 1] = m;
        }
        cl.sync();
        if (tid < 32) {  // one remote read per lane, then a shuffle max
            double m = tid < nr ? *cl.map_shared_rank(&s_max[s & 1], tid) : 0.0;
            m = warp_max(m);
            if (tid == 0) s_d = m;
        }
        __syncthreads();
        d = s_d;
        if (d < tol || s + 1 >= cap) {
            fin = s + 1;
            break;
        }
    }
    const double* res = (fin & 1) ? bufB : bufA;
    for (int e = tid; e < np * plane; e += JC_THREADS) vh[(size_t)zlo * plane + e] = res[e];
    if (r == 0 && tid == 0) {
        out->sweeps = fin;
        out->last_diff = d;
    }
    cl.sync();  // no block leaves while a neighbour may still read its shared memory
}

}  // namespace

// The whole solve inside one 16-block cluster's shared memory (grids of up to ~150k points).
// Returns false (nothing launched) when the grid does not fit or the device cannot host the cluster.
static bool hartree_cluster(dft_context* ctx, const Grid& g, const double* rho, double* vh, double tol,
                            long max_sweeps, JacobiResult* res) {
    const int nr = 16;
    const int plane = g.nx * g.ny;
    const int pmax = (g.nz + nr - 1) / nr;
    const size_t smem = sizeof(double) * 3 * (size_t)pmax * plane;
    if (g.nz < 2 * nr || smem > 200 * 1024) return false;
    static int attr_ok = -1;
    if (attr_ok < 0) {
        attr_ok = cudaFuncSetAttribute(jacobi_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
                          cudaSuccess &&
                      cudaFuncSetAttribute(jacobi_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           200 * 1024) == cudaSuccess
                  ? 1
                  : 0;
        cudaGetLastError();
    }
    if (!attr_ok) return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nr);
    cfg.blockDim = dim3(JC_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = nr;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, jacobi_cluster_kernel, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return false;
    }
    JacobiClusterOut* o = (JacobiClusterOut*)ws_get(ctx, WS_CTRL, sizeof(JacobiClusterOut) + 64);
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    DFT_CUDA(cudaLaunchKernelEx(&cfg, jacobi_cluster_kernel, g, rho, vh, o, den, tol, (long long)max_sweeps, pmax));
    count_launch(ctx);
    JacobiClusterOut* h = (JacobiClusterOut*)pinned(ctx, (sizeof(JacobiClusterOut) + 7) / 8);
    DFT_CUDA(cudaMemcpyAsync(h, o, sizeof(JacobiClusterOut), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    *res = {(long)h->sweeps, h->last_diff};
    return true;
}

// The whole solve in one cooperative launch (small grids).
static JacobiResult hartree_persistent(dft_context* ctx, const Grid& g, const double* rho, double* vh, double* buf1,
                                       double tol, long max_sweeps) {
    JacobiPCtrl* ctrl = (JacobiPCtrl*)ws_get(ctx, WS_CTRL, sizeof(JacobiPCtrl) + 64);
    DFT_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(JacobiPCtrl), ctx->stream));
    int per_sm = 0;
    DFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_persistent_kernel, 256, 0));
    const long long want = (g.N + 255) / 256;
    const int nblocks = (int)std::max<long long>(1, std::min<long long>(want, (long long)per_sm * ctx->num_sms));
    double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    long long cap = max_sweeps;
    Grid gg = g;
    const double* r = rho;
    double* b0 = vh;
    double* b1 = buf1;
    long long polls = ctx->grid_barrier_poll_limit > 0 ? ctx->grid_barrier_poll_limit : (1LL << 24);
    void* args[] = {&gg, &r, &b0, &b1, &ctrl, &den, &tol, &cap, &polls};
    DFT_CUDA(cudaLaunchCooperativeKernel((const void*)jacobi_persistent_kernel, dim3(nblocks), dim3(256), args, 0,
                                         ctx->stream));
    count_launch(ctx);
    JacobiPCtrl* hc = (JacobiPCtrl*)pinned(ctx, (sizeof(JacobiPCtrl) + 7) / 8);
    DFT_CUDA(cudaMemcpyAsync(hc, ctrl, sizeof(JacobiPCtrl), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    if (hc->error) fail(DFT_CUDA_ERROR, "Jacobi grid barrier timed out");
    if (hc->sweeps & 1)
        DFT_CUDA(cudaMemcpyAsync(vh, buf1, sizeof(double) * (size_t)g.N, cudaMemcpyDeviceToDevice, ctx->stream));
    return {(long)hc->sweeps, hc->last_diff};
}

// Jacobi with up to `tmax` sweeps per launch (2, 4 or 8), bit-identical to the one-sweep path.
static JacobiResult hartree_tb(dft_context* ctx, const Grid& g, const double* rho, double* vh, double* buf1,
                               double tol, long max_sweeps, int tmax) {
    JacobiTBCtrl* ctrl = (JacobiTBCtrl*)ws_get(ctx, WS_CTRL, sizeof(JacobiTBCtrl) + 64);
    DFT_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(JacobiTBCtrl), ctx->stream));
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    const int tt = TB_R - 2 * tmax;
    const int bx = (g.nx + tt - 1) / tt, by = (g.ny + tt - 1) / tt;
    int zc = 64;
    while (zc > 8 && (long long)bx * by * ((g.nz + zc - 1) / zc) < 2LL * ctx->num_sms) zc >>= 1;
    zc = std::max(zc, std::min(g.nz, 2 * tmax));
    dim3 grid(bx, by, (g.nz + zc - 1) / zc), block(TB_R, TB_R);
    const size_t smem = sizeof(double) * (size_t)tmax * 3 * TB_R * TB_R;
    auto launch = [&](int tsw, int replay_parity) {
        if (tmax == 2)
            jacobi_tb_kernel<2><<<grid, block, smem, ctx->stream>>>(g, rho, vh, buf1, ctrl, den, tol, max_sweeps, zc,
                                                                    tsw, replay_parity);
        else if (tmax == 4)
            jacobi_tb_kernel<4><<<grid, block, smem, ctx->stream>>>(g, rho, vh, buf1, ctrl, den, tol, max_sweeps, zc,
                                                                    tsw, replay_parity);
        else
            jacobi_tb_kernel<8><<<grid, block, smem, ctx->stream>>>(g, rho, vh, buf1, ctrl, den, tol, max_sweeps, zc,
                                                                    tsw, replay_parity);
    };
    static bool attr[3] = {false, false, false};
    const int ai = tmax == 2 ? 0 : (tmax == 4 ? 1 : 2);
    if (!attr[ai]) {
        if (tmax == 2)
            DFT_CUDA(cudaFuncSetAttribute(jacobi_tb_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        else if (tmax == 4)
            DFT_CUDA(cudaFuncSetAttribute(jacobi_tb_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        else
            DFT_CUDA(cudaFuncSetAttribute(jacobi_tb_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr[ai] = true;
    }
    JacobiTBCtrl* hc = (JacobiTBCtrl*)pinned(ctx, (sizeof(JacobiTBCtrl) + 7) / 8);
    long sweeps_launched = 0, batch = 8;
    while (true) {
        long nl = 0;
        while (nl < batch && sweeps_launched < max_sweeps) {
            launch(tmax, -1);
            sweeps_launched += tmax;
            ++nl;
        }
        DFT_LAUNCH_CHECK();
        count_launch(ctx, nl);
        DFT_CUDA(cudaMemcpyAsync(hc, ctrl, sizeof(JacobiTBCtrl), cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        if (hc->done || sweeps_launched >= max_sweeps) break;
        batch = std::min<long>(batch * 2, 256);
    }
    if (!hc->done) fail(DFT_CAP_REACHED, "Jacobi control state inconsistent");
    int out_parity = hc->final_in_parity ^ 1;  // the output buffer of the final launch
    if (hc->final_level < tmax) {
        // the stop rule fired inside the launch: recompute from its input with fewer levels
        launch(hc->final_level, hc->final_in_parity);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
    if (out_parity == 1)
        DFT_CUDA(cudaMemcpyAsync(vh, buf1, sizeof(double) * (size_t)g.N, cudaMemcpyDeviceToDevice, ctx->stream));
    return {(long)hc->sweep, hc->last_diff};
}

bool faces_exact(const Grid& g) {
    return (g.xmin + (double)(g.nx - 1) * g.dx == g.xmax) && (g.ymin + (double)(g.ny - 1) * g.dy == g.ymax) &&
           (g.zmin + (double)(g.nz - 1) * g.dz == g.zmax);
}

JacobiResult hartree(dft_context* ctx, const Grid& g, const double* rho, double* vh, double tol, long max_sweeps,
                     const double* guess, bool zero_faces) {
    if (max_sweeps < 0) fail(DFT_INVALID_ARGUMENT, "max_sweeps must be >= 0");
    double* buf1 = (double*)ws_get(ctx, WS_JACOBI, sizeof(double) * (size_t)g.N);
    JacobiCtrl* ctrl = (JacobiCtrl*)ws_get(ctx, WS_CTRL, sizeof(JacobiCtrl) + 64);
    // Boundary values are Q/|r| only on faces whose last node misses the bound by rounding
    // (reference :60-79); on every grid whose x_{n-1} == xmax they are all zero and Q is unused.
    // zero_faces forces the zero boundary (Q = 0) whatever the rounding.
    const bool exact_faces = zero_faces || faces_exact(g);
    double Q = 0.0;
    if (!exact_faces) {
        double* q = (double*)ws_get(ctx, WS_TMP2, sizeof(double));
        total_charge_seq_kernel<<<1, 32, 0, ctx->stream>>>(g.N, rho, g.dV, q);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        double* h = pinned(ctx, 1);
        DFT_CUDA(cudaMemcpyAsync(h, q, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        Q = h[0];
    }
    jacobi_init_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g, Q, vh, buf1, guess);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    DFT_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(JacobiCtrl), ctx->stream));
    if (max_sweeps == 0 || g.nx < 3 || g.ny < 3 || g.nz < 3) {
        // no interior: the reference still runs its sweep loop, finds max|dV| = 0 < tol and stops
        return {max_sweeps == 0 ? 0L : 1L, 0.0};
    }
    // launch shape: one persistent launch on small grids (launch-latency bound), one sweep per
    // launch otherwise; 2/4/8 select the temporally blocked kernel
    int tmax = ctx->jacobi_sweeps_per_launch;
    if (tmax == 0) {
        auto t = ctx->tuned.find({(long long)g.nx, (long long)g.ny, (long long)g.nz});
        if (t != ctx->tuned.end()) tmax = t->second[1];
    }
    if (tmax == 0 || tmax == -2) {
        JacobiResult r;
        if (hartree_cluster(ctx, g, rho, vh, tol, max_sweeps, &r)) return r;
        if (tmax == -2) fail(DFT_INVALID_ARGUMENT, "grid does not fit the cluster-resident Jacobi");
    }
    if (tmax == 0) tmax = g.N <= 64LL * 64 * 64 ? -1 : 1;
    if (tmax == -1) return hartree_persistent(ctx, g, rho, vh, buf1, tol, max_sweeps);
    if (tmax == 2 || tmax == 4 || tmax == 8) return hartree_tb(ctx, g, rho, vh, buf1, tol, max_sweeps, tmax);
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    dim3 block(JB_X, JB_Y);
    const int bx = (g.nx + JB_X - 1) / JB_X, by = (g.ny + JB_Y - 1) / JB_Y;
    int zc = 32;
    while (zc > 4 && (long long)bx * by * ((g.nz + zc - 1) / zc) < 2LL * ctx->num_sms) zc >>= 1;
    dim3 grid(bx, by, (g.nz + zc - 1) / zc);
    JacobiCtrl* hc = (JacobiCtrl*)pinned(ctx, (sizeof(JacobiCtrl) + 7) / 8);
    long launched = 0;
    // Sweeps are launched in batches; a launch after the stop rule fired returns at once, so
    // a batch may overrun the stopping sweep without changing the result.
    long batch = 32;
    while (true) {
        const long nb = std::min<long>(batch, max_sweeps - launched);
        for (long s = 0; s < nb; ++s) {
            jacobi_sweep_kernel<<<grid, block, 0, ctx->stream>>>(g, rho, vh, buf1, ctrl, den, tol, max_sweeps, zc);
        }
        DFT_LAUNCH_CHECK();
        count_launch(ctx, nb);
        launched += nb;
        DFT_CUDA(cudaMemcpyAsync(hc, ctrl, sizeof(JacobiCtrl), cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        if (hc->done || launched >= max_sweeps) break;
        batch = std::min<long>(batch * 2, 512);
    }
    const long sweeps = (long)hc->sweep;
    if (sweeps & 1) {
        DFT_CUDA(cudaMemcpyAsync(vh, buf1, sizeof(double) * (size_t)g.N, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return {sweeps, hc->last_diff};
}

// =============================================================== monopole boundary (option)
// The reference's face values are Q/|r| (|r| from the origin, Q the total charge), except that
// a face whose last node lands exactly on the bound gets 0 (HartreePotentialMolecule.cpp:45-94);
// every grid of the benchmark systems lands exactly, so their faces are all 0.  For many
// electrons the zero faces are far from the free-space potential and bind spurious states at
// the box walls.  The option applies Q/|r| on every face.  It is solved without touching the
// zero-face solvers: with V_c = Q erf(|r| / (sqrt(2) s)) / |r| (which equals Q/|r| on the faces
// to double precision for s <= face distance / 8), V_H = V' + V_c where V' has zero faces and
// L_h V' = -4 pi rho - L_h V_c, L_h the same 7-point Laplacian: the discrete problem is exactly
// the Dirichlet problem with V_c's face values.
namespace {
struct SumF {
    const double* a;
    __device__ void operator()(long long p, double* acc) const { acc[0] += a[p]; }
};

__device__ __forceinline__ double gauss_pot(double q, double s, double r) {
    // q erf(r / (sqrt(2) s)) / r, its limit q sqrt(2/pi) / s at r = 0
    if (r < 1e-10 * s) return q * 0.79788456080286535588 / s;
    return q * erf(r * (0.70710678118654752440 / s)) / r;
}

__global__ void monopole_comp_kernel(Grid g, double q, double s, double* __restrict__ vc) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const double x = g.xmin + i * g.dx, y = g.ymin + j * g.dy, z = g.zmin + k * g.dz;
        vc[p] = gauss_pot(q, s, sqrt(x * x + y * y + z * z));
    }
}

// interior: out = rho + (L_h vc) / (4 pi); faces: 0 (unused by the solvers)
__global__ void monopole_source_kernel(Grid g, const double* __restrict__ rho, const double* __restrict__ vc,
                                       double* __restrict__ out) {
    const double inv4pi = 1.0 / (4.0 * xcf::PI);
    const long long sxy = (long long)g.nx * g.ny;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / sxy);
        if (i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz) {
            out[p] = 0.0;
            continue;
        }
        const double c = vc[p];
        const double lap = g.ix2 * (vc[p - 1] + vc[p + 1] - 2.0 * c) + g.iy2 * (vc[p - g.nx] + vc[p + g.nx] - 2.0 * c) +
                           g.iz2 * (vc[p - sxy] + vc[p + sxy] - 2.0 * c);
        out[p] = rho[p] + lap * inv4pi;
    }
}

__global__ void add_into_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b,
                                double* __restrict__ o) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        o[p] = a[p] + b[p];
}
}  // namespace

double monopole_width(const Grid& g) {
    const double d = std::min({-g.xmin, g.xmax, -g.ymin, g.ymax, -g.zmin, g.zmax});
    if (!(d > 4.0 * std::max({g.dx, g.dy, g.dz})))
        fail(DFT_INVALID_ARGUMENT, "the monopole boundary needs the origin well inside the box");
    return d / 8.0;
}

double monopole_prepare(dft_context* ctx, const Grid& g, const double* rho, double* rho_prime, double* vc) {
    double q = 0.0;
    reduce_to_host<1>(ctx, g.N, SumF{rho}, &q);
    q *= g.dV;
    const double s = monopole_width(g);
    monopole_comp_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g, q, s, vc);
    monopole_source_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g, rho, vc, rho_prime);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    return q;
}

namespace {
__global__ void zero_faces_kernel(Grid g, double* __restrict__ v) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        if (i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz) v[p] = 0.0;
    }
}
}  // namespace

void zero_faces(dft_context* ctx, const Grid& g, double* v) {
    zero_faces_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g, v);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void add_into(dft_context* ctx, long long n, const double* a, const double* b, double* out) {
    add_into_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, a, b, out);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

// =============================================================== allocation-free Poisson
// The Jacobi solve above takes its second iterate buffer and its control words from the
// context's workspace, which grows with cudaMalloc.  Some callers cannot let a library
// allocate device memory: a host application that owns the whole device memory budget
// through its own pooled allocator, or a plugin called from inside such an application's
// compute step, where a cudaMalloc/cudaFree would also synchronise the device.  For them
// hartree_noalloc runs the same kernels on a fixed scratch array compiled into the library.
//
// Limit: grids of at most NOALLOC_MAX_POINTS points (128^3).  Every GPU on which a context
// is created holds the array (16 MiB + 128 B) until the process exits: dft_context_create
// looks up its address, which also makes CUDA load this file's module (and the array) when
// modules load lazily, so the first allocation-free call does not load it in the middle of
// the caller's compute step.  All calls share the array: calls that overlap on the GPU
// (several streams or contexts on one device) race on it.  Each call runs one Jacobi sweep
// per launch (jacobi_sweep_kernel), whatever jacobi_sweeps_per_launch says: the cluster and
// persistent variants take further workspace.
namespace {

constexpr long long NOALLOC_MAX_POINTS = 128LL * 128 * 128;
constexpr int NOALLOC_CTRL_DOUBLES = 16;  // JacobiCtrl and the boundary charge live after the buffer

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_POINTS + NOALLOC_CTRL_DOUBLES];

static_assert(sizeof(JacobiCtrl) + sizeof(double) <= NOALLOC_CTRL_DOUBLES * sizeof(double), "control words");

}  // namespace

// Device address of g_noalloc_scratch, looked up once per device with that device current.
double* noalloc_scratch(int device) {
    static double* addr[64] = {};
    static std::mutex m;
    if (device < 0 || device >= 64) fail(DFT_INVALID_ARGUMENT, "device index %d out of range", device);
    std::lock_guard<std::mutex> lock(m);
    if (!addr[device]) {
        double* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            fail(DFT_CUDA_ERROR, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(e));
        addr[device] = p;
    }
    return addr[device];
}

JacobiResult hartree_noalloc(dft_context* ctx, const Grid& g, const double* rho, double* vh, double tol,
                             long max_sweeps) {
    if (g.N > NOALLOC_MAX_POINTS)
        fail(DFT_INVALID_ARGUMENT,
             "grid of %lld points exceeds the allocation-free Poisson limit of %lld points (128^3); "
             "use dft_hartree_dev",
             g.N, NOALLOC_MAX_POINTS);
    if (max_sweeps < 0) fail(DFT_INVALID_ARGUMENT, "max_sweeps must be >= 0");
    double* scratch = noalloc_scratch(ctx->device);
    double* buf1 = scratch;
    JacobiCtrl* ctrl = (JacobiCtrl*)(scratch + NOALLOC_MAX_POINTS);
    double* qslot = scratch + NOALLOC_MAX_POINTS + NOALLOC_CTRL_DOUBLES - 1;
    double Q = 0.0;
    if (!faces_exact(g)) {
        total_charge_seq_kernel<<<1, 32, 0, ctx->stream>>>(g.N, rho, g.dV, qslot);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        DFT_CUDA(cudaMemcpyAsync(&Q, qslot, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
    }
    jacobi_init_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g, Q, vh, buf1, nullptr);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    // the array keeps the previous call's control words: clear them
    DFT_CUDA(cudaMemsetAsync(ctrl, 0, sizeof(JacobiCtrl), ctx->stream));
    if (max_sweeps == 0 || g.nx < 3 || g.ny < 3 || g.nz < 3) {
        sync(ctx);
        return {max_sweeps == 0 ? 0L : 1L, 0.0};
    }
    const double den = 2.0 * (g.ix2 + g.iy2 + g.iz2);
    dim3 block(JB_X, JB_Y);
    const int bx = (g.nx + JB_X - 1) / JB_X, by = (g.ny + JB_Y - 1) / JB_Y;
    int zc = 32;
    while (zc > 4 && (long long)bx * by * ((g.nz + zc - 1) / zc) < 2LL * ctx->num_sms) zc >>= 1;
    dim3 grid(bx, by, (g.nz + zc - 1) / zc);
    JacobiCtrl hc;
    long launched = 0, batch = 32;
    while (true) {
        const long nb = std::min<long>(batch, max_sweeps - launched);
        for (long s = 0; s < nb; ++s)
            jacobi_sweep_kernel<<<grid, block, 0, ctx->stream>>>(g, rho, vh, buf1, ctrl, den, tol, max_sweeps, zc);
        DFT_LAUNCH_CHECK();
        count_launch(ctx, nb);
        launched += nb;
        DFT_CUDA(cudaMemcpyAsync(&hc, ctrl, sizeof(JacobiCtrl), cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        if (hc.done || launched >= max_sweeps) break;
        batch = std::min<long>(batch * 2, 512);
    }
    const long sweeps = (long)hc.sweep;
    if (sweeps & 1)
        DFT_CUDA(cudaMemcpyAsync(vh, buf1, sizeof(double) * (size_t)g.N, cudaMemcpyDeviceToDevice, ctx->stream));
    sync(ctx);
    return {sweeps, hc.last_diff};
}

// =============================================================== XC ==================
namespace {

// Pass 1: functional at every point above the floor.  Writes d f/d n_sigma and the gradient
// coefficients c_sigma (zero below the floor, reference :626-706) and per-block partial sums
// of n eps dV (reference :749-842).  One evaluation serves both spins and the energy.
template <int KIND, bool POT, bool ENERGY>
__global__ void __launch_bounds__(256) xc_point_kernel(Grid g, const double* __restrict__ na,
                                                       const double* __restrict__ nb, double* __restrict__ da,
                                                       double* __restrict__ db, double* __restrict__ ca,
                                                       double* __restrict__ cb, double* __restrict__ partial) {
    __shared__ double sh[8];
    double e = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const double a = na[p], b = nb[p];
        const double n = a + b;
        double rda = 0.0, rdb = 0.0, rca = 0.0, rcb = 0.0;
        if (n > xcf::RHO_FLOOR) {
            const int i = (int)(p % g.nx);
            const int j = (int)((p / g.nx) % g.ny);
            const int k = (int)(p / ((long long)g.nx * g.ny));
            double ga = 0.0, gb = 0.0;
            if (KIND == 1) {
                ga = gradmag(g, na, p, i, j, k);
                gb = gradmag(g, nb, p, i, j, k);
            }
            const xcf::Result r = xcf::evaluate<KIND>(a, b, ga, gb);
            rda = r.va;
            rdb = r.vb;
            rca = r.ca;
            rcb = r.cb;
            if (ENERGY) e += n * r.eps * g.dV;
        }
        if (POT) {
            da[p] = rda;
            db[p] = rdb;
            if (KIND == 1) {
                ca[p] = rca;
                cb[p] = rcb;
            }
        }
    }
    if (ENERGY) {
        e = block_sum(e, sh);
        if (threadIdx.x == 0) partial[blockIdx.x] = e;
    }
}

// div(c grad f) at (i,j,k), reference calculateCartesianDivergence :216-572
__device__ __forceinline__ double ddiv(const Grid& g, const double* __restrict__ c, const double* __restrict__ f,
                                       long long p, int i, int j, int k) {
    const double cc = c[p];
    double dx, dy, dz;
    {
        const double fc = cc * dderiv(g, f, p, i, j, k, 0);
        if (i == 0) dx = (c[p + 1] * dderiv(g, f, p + 1, i + 1, j, k, 0) - fc) / g.dx;
        else if (i == g.nx - 1) dx = (fc - c[p - 1] * dderiv(g, f, p - 1, i - 1, j, k, 0)) / g.dx;
        else
            dx = (c[p + 1] * dderiv(g, f, p + 1, i + 1, j, k, 0) - c[p - 1] * dderiv(g, f, p - 1, i - 1, j, k, 0)) /
                 (2.0 * g.dx);
    }
    {
        const long long s = g.nx;
        const double fc = cc * dderiv(g, f, p, i, j, k, 1);
        if (j == 0) dy = (c[p + s] * dderiv(g, f, p + s, i, j + 1, k, 1) - fc) / g.dy;
        else if (j == g.ny - 1) dy = (fc - c[p - s] * dderiv(g, f, p - s, i, j - 1, k, 1)) / g.dy;
        else
            dy = (c[p + s] * dderiv(g, f, p + s, i, j + 1, k, 1) - c[p - s] * dderiv(g, f, p - s, i, j - 1, k, 1)) /
                 (2.0 * g.dy);
    }
    {
        const long long s = (long long)g.nx * g.ny;
        const double fc = cc * dderiv(g, f, p, i, j, k, 2);
        if (k == 0) dz = (c[p + s] * dderiv(g, f, p + s, i, j, k + 1, 2) - fc) / g.dz;
        else if (k == g.nz - 1) dz = (fc - c[p - s] * dderiv(g, f, p - s, i, j, k - 1, 2)) / g.dz;
        else
            dz = (c[p + s] * dderiv(g, f, p + s, i, j, k + 1, 2) - c[p - s] * dderiv(g, f, p - s, i, j, k - 1, 2)) /
                 (2.0 * g.dz);
    }
    return dx + dy + dz;
}

// Pass 2 (GGA only): v_sigma = d_sigma - div(c_sigma grad n_sigma) above the floor, else 0.
__global__ void __launch_bounds__(256) xc_div_kernel(Grid g, const double* __restrict__ na,
                                                     const double* __restrict__ nb, const double* __restrict__ da,
                                                     const double* __restrict__ db, const double* __restrict__ ca,
                                                     const double* __restrict__ cb, double* __restrict__ va,
                                                     double* __restrict__ vb) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const double n = na[p] + nb[p];
        double ra = 0.0, rb = 0.0;
        if (n > xcf::RHO_FLOOR) {
            const int i = (int)(p % g.nx);
            const int j = (int)((p / g.nx) % g.ny);
            const int k = (int)(p / ((long long)g.nx * g.ny));
            if (va) ra = da[p] - ddiv(g, ca, na, p, i, j, k);
            if (vb) rb = db[p] - ddiv(g, cb, nb, p, i, j, k);
        }
        if (va) va[p] = ra;
        if (vb) vb[p] = rb;
    }
}

// LDA potential: the divergence term vanishes identically (c = 0), v = d above the floor.
__global__ void xc_lda_copy_kernel(long long n, const double* __restrict__ na, const double* __restrict__ nb,
                                   const double* __restrict__ da, const double* __restrict__ db, double* va,
                                   double* vb) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const bool on = na[p] + nb[p] > xcf::RHO_FLOOR;
        if (va) va[p] = on ? da[p] : 0.0;
        if (vb) vb[p] = on ? db[p] : 0.0;
    }
}

template <int KIND>
__global__ void xc_eval_kernel(long long m, const double* na, const double* nb, const double* ga, const double* gb,
                               double* out5) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < m; p += (long long)gridDim.x * blockDim.x) {
        const xcf::Result r = xcf::evaluate<KIND>(na[p], nb[p], ga[p], gb[p]);
        out5[5 * p + 0] = r.eps;
        out5[5 * p + 1] = r.va;
        out5[5 * p + 2] = r.vb;
        out5[5 * p + 3] = r.ca;
        out5[5 * p + 4] = r.cb;
    }
}

template <int KIND>
double xc_impl(dft_context* ctx, const Grid& g, const double* na, const double* nb, double* va, double* vb,
               bool want_energy) {
    const bool pot = va || vb;
    const size_t N = (size_t)g.N;
    double* tmp = pot ? (double*)ws_get(ctx, WS_XC, sizeof(double) * 4 * N) : nullptr;
    double *da = tmp, *db = tmp ? tmp + N : nullptr, *ca = tmp ? tmp + 2 * N : nullptr, *cb = tmp ? tmp + 3 * N : nullptr;
    const int nbk = std::max(1, std::min((int)((g.N + 255) / 256), ctx->num_sms * 8));
    double* partial = (double*)ws_get(ctx, WS_REDUCE, sizeof(double) * ((size_t)nbk + 8));
    if (pot && want_energy)
        xc_point_kernel<KIND, true, true><<<nbk, 256, 0, ctx->stream>>>(g, na, nb, da, db, ca, cb, partial);
    else if (pot)
        xc_point_kernel<KIND, true, false><<<nbk, 256, 0, ctx->stream>>>(g, na, nb, da, db, ca, cb, partial);
    else
        xc_point_kernel<KIND, false, true><<<nbk, 256, 0, ctx->stream>>>(g, na, nb, da, db, ca, cb, partial);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    if (pot) {
        if (KIND == 1)
            xc_div_kernel<<<nbk, 256, 0, ctx->stream>>>(g, na, nb, da, db, ca, cb, va, vb);
        else
            xc_lda_copy_kernel<<<nbk, 256, 0, ctx->stream>>>(g.N, na, nb, da, db, va, vb);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
    if (!want_energy) return 0.0;
    double* res = partial + nbk;
    reduce_final_kernel<1><<<1, 256, 0, ctx->stream>>>(nbk, partial, res);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    double* h = pinned(ctx, 1);
    DFT_CUDA(cudaMemcpyAsync(h, res, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    return h[0];
}

}  // namespace

double xc(dft_context* ctx, const Grid& g, int kind, const double* na, const double* nb, double* va, double* vb,
          bool want_energy) {
    if (kind == DFT_XC_PBE96) return xc_impl<1>(ctx, g, na, nb, va, vb, want_energy);
    if (kind == DFT_XC_PZ81) return xc_impl<0>(ctx, g, na, nb, va, vb, want_energy);
    fail(DFT_INVALID_ARGUMENT, "unknown functional kind %d", kind);
}

void xc_evaluate(dft_context* ctx, int kind, long long m, const double* na, const double* nb, const double* ga,
                 const double* gb, double* out5) {
    if (m <= 0) return;
    const int nbk = std::max(1, std::min((int)((m + 255) / 256), ctx->num_sms * 8));
    if (kind == DFT_XC_PBE96) xc_eval_kernel<1><<<nbk, 256, 0, ctx->stream>>>(m, na, nb, ga, gb, out5);
    else if (kind == DFT_XC_PZ81) xc_eval_kernel<0><<<nbk, 256, 0, ctx->stream>>>(m, na, nb, ga, gb, out5);
    else fail(DFT_INVALID_ARGUMENT, "unknown functional kind %d", kind);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

// =============================================================== density / energies ==
namespace {

constexpr int MAX_OCC_BANDS = 1024;
struct OccTable {
    double w[MAX_OCC_BANDS];
};

// reference ElectronDensityMolecule.cpp:58-71: density += electrons * psi * psi, band order
__global__ void density_kernel(long long n, const double* __restrict__ psi, int nbands, long long ld, OccTable occ,
                               double* __restrict__ out) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        double d = 0.0;
        for (int b = 0; b < nbands; ++b) {
            const double w = occ.w[b];
            if (w <= 0.0) continue;
            const double v = psi[(long long)b * ld + p];
            d = __dadd_rn(d, __dmul_rn(__dmul_rn(w, v), v));
        }
        out[p] = d;
    }
}

// Kinetic energy density with the reference's face stencil (TotalEnergyMolecule.cpp:80-177):
// lap = sum over existing neighbours (psi_nb - psi)/h^2, term = psi * (-0.5 lap) * dV.
// One block row of partials per band.
__global__ void __launch_bounds__(256) kinetic_kernel(Grid g, const double* __restrict__ psi, long long ld,
                                                      double* partial) {
    __shared__ double sh[8];
    const int band = blockIdx.y;
    const double* __restrict__ f = psi + (long long)band * ld;
    const double hx = g.dx * g.dx, hy = g.dy * g.dy, hz = g.dz * g.dz;
    const long long sxy = (long long)g.nx * g.ny;
    double e = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx);
        const int j = (int)((p / g.nx) % g.ny);
        const int k = (int)(p / sxy);
        const double c = f[p];
        double lap = 0.0;
        if (i > 0) lap += (f[p - 1] - c) / hx;
        if (i + 1 < g.nx) lap += (f[p + 1] - c) / hx;
        if (j > 0) lap += (f[p - g.nx] - c) / hy;
        if (j + 1 < g.ny) lap += (f[p + g.nx] - c) / hy;
        if (k > 0) lap += (f[p - sxy] - c) / hz;
        if (k + 1 < g.nz) lap += (f[p + sxy] - c) / hz;
        e += c * (-0.5 * lap) * g.dV;
    }
    e = block_sum(e, sh);
    if (threadIdx.x == 0) partial[(long long)band * gridDim.x + blockIdx.x] = e;
}

__global__ void rows_sum_kernel(int nrows, int ncols, const double* partial, double* out) {
    __shared__ double sh[32];
    for (int r = 0; r < nrows; ++r) {
        double s = 0.0;
        for (int c = threadIdx.x; c < ncols; c += blockDim.x) s += partial[(long long)r * ncols + c];
        s = block_sum(s, sh);
        if (threadIdx.x == 0) out[r] = s;
    }
}

// NuclearPotential::calculateAtPoint, reference NuclearPotential.cpp:36-76
__global__ void nuclear_kernel(Grid g, int nnuc, const double* __restrict__ nuc, double* __restrict__ v,
                               int* singular) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx);
        const int j = (int)((p / g.nx) % g.ny);
        const int k = (int)(p / ((long long)g.nx * g.ny));
        const double x = __dadd_rn(g.xmin, __dmul_rn((double)i, g.dx));
        const double y = __dadd_rn(g.ymin, __dmul_rn((double)j, g.dy));
        const double z = __dadd_rn(g.zmin, __dmul_rn((double)k, g.dz));
        double s = 0.0;
        for (int a = 0; a < nnuc; ++a) {
            const double ddx = x - nuc[4 * a + 1], ddy = y - nuc[4 * a + 2], ddz = z - nuc[4 * a + 3];
            const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
            if (d2 == 0.0) {
                atomicExch(singular, 1);
                continue;
            }
            s = __dsub_rn(s, __ddiv_rn(nuc[4 * a], sqrt(d2)));
        }
        v[p] = s;
    }
}

}  // namespace

void spin_density(dft_context* ctx, long long n, const double* psi, int nbands, long long ld, const double* occ_host,
                  double* out) {
    if (nbands > MAX_OCC_BANDS) fail(DFT_INVALID_ARGUMENT, "at most %d bands", MAX_OCC_BANDS);
    OccTable t;
    for (int b = 0; b < nbands; ++b) t.w[b] = occ_host[b];
    density_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, psi, nbands, ld, t, out);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void kinetic_per_band(dft_context* ctx, const Grid& g, const double* psi, int nbands, long long ld, double* out_host) {
    if (nbands <= 0) return;
    if (nbands > 65535) fail(DFT_INVALID_ARGUMENT, "too many bands");
    const int nbk = std::max(1, std::min((int)((g.N + 255) / 256), ctx->num_sms * 2));
    double* partial = (double*)ws_get(ctx, WS_REDUCE, sizeof(double) * ((size_t)nbk * nbands + nbands));
    double* res = partial + (size_t)nbk * nbands;
    kinetic_kernel<<<dim3(nbk, nbands), 256, 0, ctx->stream>>>(g, psi, ld, partial);
    DFT_LAUNCH_CHECK();
    rows_sum_kernel<<<1, 256, 0, ctx->stream>>>(nbands, nbk, partial, res);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    double* h = pinned(ctx, nbands);
    DFT_CUDA(cudaMemcpyAsync(h, res, sizeof(double) * nbands, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    for (int b = 0; b < nbands; ++b) out_host[b] = h[b];
}

double kinetic_energy(dft_context* ctx, const Grid& g, const double* psi, int nbands, long long ld,
                      const double* occ_host) {
    std::vector<double> e(std::max(nbands, 1));
    kinetic_per_band(ctx, g, psi, nbands, ld, e.data());
    // energy += electrons * orbitalEnergy, in band order (reference TotalEnergyMolecule.cpp:181-195)
    double s = 0.0;
    for (int b = 0; b < nbands; ++b)
        if (occ_host[b] > 0.0) s += occ_host[b] * e[b];
    return s;
}

void nuclear_potential(dft_context* ctx, const Grid& g, int nnuc, const int* Z, const double* xyz, double* vext) {
    if (nnuc <= 0) fail(DFT_INVALID_ARGUMENT, "La molecula debe contener al menos un nucleo.");
    std::vector<double> nuc(4 * (size_t)nnuc);
    for (int a = 0; a < nnuc; ++a) {
        if (Z[a] <= 0) fail(DFT_INVALID_ARGUMENT, "Atomic number must be greater than zero.");
        nuc[4 * a] = (double)Z[a];
        nuc[4 * a + 1] = xyz[3 * a];
        nuc[4 * a + 2] = xyz[3 * a + 1];
        nuc[4 * a + 3] = xyz[3 * a + 2];
    }
    double* dn = (double*)ws_get(ctx, WS_TMP2, sizeof(double) * nuc.size() + 64);
    int* flag = (int*)(dn + nuc.size());
    DFT_CUDA(cudaMemcpyAsync(dn, nuc.data(), sizeof(double) * nuc.size(), cudaMemcpyHostToDevice, ctx->stream));
    DFT_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream));
    nuclear_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g, nnuc, dn, vext, flag);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    int* h = (int*)pinned(ctx, 1);
    DFT_CUDA(cudaMemcpyAsync(h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    if (*h) fail(DFT_SINGULAR, "NuclearPotential is singular at a nuclear position.");
}


// =============================================================== Pulay mixing support
namespace {
struct LinComb {
    const double* a[16];
    const double* r[16];
    double c[16];
    int m;
};
// out = max(0, sum_i c_i (a_i + beta r_i))
__global__ void lincomb_kernel(long long n, LinComb L, double beta, double* __restrict__ out) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < L.m; ++i) s += L.c[i] * (L.a[i][p] + beta * L.r[i][p]);
        out[p] = s > 0.0 ? s : 0.0;
    }
}
__global__ void sub_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ out) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        out[p] = a[p] - b[p];
}
// out = sum_i c_i a_i (no clamp)
__global__ void combine_kernel(long long n, LinComb L, double* __restrict__ out) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < L.m; ++i) s += L.c[i] * L.a[i][p];
        out[p] = s;
    }
}
// out = max(0, a + beta (r - f x)); out may alias a
__global__ void kerker_update_kernel(long long n, const double* a, const double* __restrict__ r,
                                     const double* __restrict__ x, double f, double beta, double* out) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const double v = a[p] + beta * (r[p] - f * x[p]);
        out[p] = v > 0.0 ? v : 0.0;
    }
}
__global__ void add2_plain_kernel(long long n, const double* __restrict__ a, const double* __restrict__ b,
                                  double* __restrict__ o) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        o[p] = a[p] + b[p];
}
}  // namespace

void combine(dft_context* ctx, long long n, int m, const double* const* a, const double* c, double* out) {
    if (m < 1 || m > 16) fail(DFT_INVALID_ARGUMENT, "combination of %d entries", m);
    LinComb L{};
    L.m = m;
    for (int i = 0; i < m; ++i) {
        L.a[i] = a[i];
        L.c[i] = c[i];
    }
    combine_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, L, out);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void kerker_update(dft_context* ctx, const Grid& g, int ns, double* const* a, const double* const* r, double* rtot,
                   double* x, double q2, double beta) {
    if (ns == 2) {
        add2_plain_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g.N, r[0], r[1], rtot);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
    // closed shell: the total residual is 2 r, so (q^2/2) V(2 r) = q^2 V(r)
    screened_poisson_vcycle(ctx, g, ns == 2 ? rtot : r[0], 1, q2, x, g.N, 2);
    const double f = ns == 2 ? 0.5 * q2 : q2;
    for (int sp = 0; sp < ns; ++sp) {
        kerker_update_kernel<<<ew_blocks(ctx, g.N), 256, 0, ctx->stream>>>(g.N, a[sp], r[sp], x, f, beta, a[sp]);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
    }
}

void pulay_combine(dft_context* ctx, long long n, int m, const double* const* a, const double* const* r,
                   const double* c, double beta, double* out) {
    if (m < 1 || m > 16) fail(DFT_INVALID_ARGUMENT, "Pulay history of %d entries", m);
    LinComb L{};
    L.m = m;
    for (int i = 0; i < m; ++i) {
        L.a[i] = a[i];
        L.r[i] = r[i];
        L.c[i] = c[i];
    }
    lincomb_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, L, beta, out);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void sub(dft_context* ctx, long long n, const double* a, const double* b, double* out) {
    sub_kernel<<<ew_blocks(ctx, n), 256, 0, ctx->stream>>>(n, a, b, out);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

}  // namespace dftb
