// Learned start for the Jacobi Poisson solve: coarse-grid solve + 3D convolutional network.
// No counterpart in the reference (its solve starts from zero, HartreePotentialMolecule.cpp:152-155).
//
// Network (NDHWC activations in BF16, FP32 accumulation, FP32 master weights):
//   level 0 (fine grid)       c1: conv3 in->16   c2: conv3 16->16                 (skip s0 = a2)
//   level 1 (ceil(n/2))       c3: down 16->32    c4: conv3 32->32                 (skip s1 = a4)
//   level 2 (ceil(n/4))       c5: down 32->32    c6: conv3 32->32   c7: conv3 32->32
//   level 1                   c8: up 32->32 (+ s1)  c9: conv3 32->32
//   level 0                   c10: up 32->16 (+ s0) c11: conv3 16->16  c12: 1x1 16->1 (FP32 out)
// conv3 = 3x3x3, zero padding; down = 2x2x2 stride 2; up = 2x2x2 stride-2 transposed;
// every layer but c12 is followed by SiLU.  Weights are [tap][cin][cout], then bias[cout].
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <memory>
#include <numeric>
#include <random>
#include <vector>

#include "common.cuh"
#include "neural.h"
#include "ops.h"

namespace dftb {
namespace {

using bf16 = __nv_bfloat16;

struct Vol {
    int nx, ny, nz;
    __host__ __device__ long long n() const { return (long long)nx * ny * nz; }
};
inline Vol half_vol(Vol v) { return {(v.nx + 1) / 2, (v.ny + 1) / 2, (v.nz + 1) / 2}; }

__device__ __forceinline__ float bf_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
__device__ __forceinline__ uint32_t pack_bf2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.f + z * (1.f - s));
}

// CC channels starting at p (aligned to CC elements) as floats
template <int CC>
__device__ __forceinline__ void ldc(const bf16* p, float* f) {
    if constexpr (CC == 2) {
        const uint32_t w = *reinterpret_cast<const uint32_t*>(p);
        f[0] = bf_lo(w);
        f[1] = bf_hi(w);
    } else {
        const uint2 w = *reinterpret_cast<const uint2*>(p);
        f[0] = bf_lo(w.x);
        f[1] = bf_hi(w.x);
        f[2] = bf_lo(w.y);
        f[3] = bf_hi(w.y);
    }
}
template <int CC>
__device__ __forceinline__ void ldc(const float* p, float* f) {
    if constexpr (CC == 2) {
        const float2 w = *reinterpret_cast<const float2*>(p);
        f[0] = w.x;
        f[1] = w.y;
    } else {
        const float4 w = *reinterpret_cast<const float4*>(p);
        f[0] = w.x;
        f[1] = w.y;
        f[2] = w.z;
        f[3] = w.w;
    }
}
// C bf16 values (C % 8 == 0, 16-byte aligned) as floats
template <int C>
__device__ __forceinline__ void ldrow(const bf16* p, float* f) {
#pragma unroll
    for (int k = 0; k < C / 8; ++k) {
        const uint4 u = reinterpret_cast<const uint4*>(p)[k];
        f[8 * k + 0] = bf_lo(u.x);
        f[8 * k + 1] = bf_hi(u.x);
        f[8 * k + 2] = bf_lo(u.y);
        f[8 * k + 3] = bf_hi(u.y);
        f[8 * k + 4] = bf_lo(u.z);
        f[8 * k + 5] = bf_hi(u.z);
        f[8 * k + 6] = bf_lo(u.w);
        f[8 * k + 7] = bf_hi(u.w);
    }
}
template <int C>
__device__ __forceinline__ void ldrow(const float* p, float* f) {
#pragma unroll
    for (int k = 0; k < C / 4; ++k) {
        const float4 u = reinterpret_cast<const float4*>(p)[k];
        f[4 * k + 0] = u.x;
        f[4 * k + 1] = u.y;
        f[4 * k + 2] = u.z;
        f[4 * k + 3] = u.w;
    }
}
template <int C>
__device__ __forceinline__ void strow(bf16* p, const float* f) {
#pragma unroll
    for (int k = 0; k < C / 8; ++k) {
        uint4 u;
        u.x = pack_bf2(f[8 * k + 0], f[8 * k + 1]);
        u.y = pack_bf2(f[8 * k + 2], f[8 * k + 3]);
        u.z = pack_bf2(f[8 * k + 4], f[8 * k + 5]);
        u.w = pack_bf2(f[8 * k + 6], f[8 * k + 7]);
        reinterpret_cast<uint4*>(p)[k] = u;
    }
}

// Copies an (hx, hy, hz) box of C-channel points whose first point is (x0, y0, z0) (may lie
// outside the volume) into shared memory, zero outside the volume.
template <int C, typename T>
__device__ void load_box(const Vol v, const T* __restrict__ src, T* dst, int x0, int y0, int z0, int hx, int hy,
                         int hz, int tid, int nthreads) {
    constexpr int ROWB = C * (int)sizeof(T);
    constexpr int CB = ROWB % 16 == 0 ? 16 : (ROWB % 8 == 0 ? 8 : 4);
    constexpr int NC = ROWB / CB;
    const int total = hx * hy * hz * NC;
    for (int e = tid; e < total; e += nthreads) {
        const int c = e % NC, pt = e / NC;
        const int lx = pt % hx, ly = (pt / hx) % hy, lz = pt / (hx * hy);
        const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
        char* d = reinterpret_cast<char*>(dst + (size_t)pt * C) + c * CB;
        const bool in = gx >= 0 && gx < v.nx && gy >= 0 && gy < v.ny && gz >= 0 && gz < v.nz;
        const char* s = in ? reinterpret_cast<const char*>(src + (((long long)gz * v.ny + gy) * v.nx + gx) * C) + c * CB
                           : nullptr;
        if constexpr (CB == 16) {
            *reinterpret_cast<uint4*>(d) = in ? *reinterpret_cast<const uint4*>(s) : make_uint4(0, 0, 0, 0);
        } else if constexpr (CB == 8) {
            *reinterpret_cast<uint2*>(d) = in ? *reinterpret_cast<const uint2*>(s) : make_uint2(0, 0);
        } else {
            *reinterpret_cast<uint32_t*>(d) = in ? *reinterpret_cast<const uint32_t*>(s) : 0u;
        }
    }
}

// ---------------------------------------------------------------- 3x3x3 convolution ----
// One thread per (x, y) column of C3_P consecutive z points; block tile 16 x 8 x 4 points.
// Forward (BWD = false): z = bias + sum_tap,ci w[tap][ci][co] in[p + off(tap)][ci]; stores z
// and a = silu(z) in BF16.  Backward data (BWD = true, w = flipped/transposed weights):
// g = (sum + extra) * silu'(zprev), stored in FP32.
constexpr int C3_X = 16, C3_Y = 8, C3_P = 4, C3_THREADS = C3_X * C3_Y;
constexpr int C3_HX = C3_X + 2, C3_HY = C3_Y + 2, C3_HZ = C3_P + 2, C3_HPTS = C3_HX * C3_HY * C3_HZ;

constexpr size_t al16(size_t b) { return (b + 15) / 16 * 16; }

template <int CIN, int COUT, typename TIN>
constexpr size_t conv3_smem() {
    return al16((size_t)27 * CIN * COUT * 2) + (size_t)C3_HPTS * CIN * sizeof(TIN);
}

template <int CIN, int COUT, typename TIN, bool BWD>
__global__ void __launch_bounds__(C3_THREADS) conv3_kernel(Vol v, const TIN* __restrict__ in,
                                                           const bf16* __restrict__ w,
                                                           const float* __restrict__ bias, bf16* __restrict__ zout,
                                                           bf16* __restrict__ aout, float* __restrict__ gout,
                                                           const float* __restrict__ extra,
                                                           const bf16* __restrict__ zprev) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int WN = 27 * CIN * COUT;
    bf16* ws = reinterpret_cast<bf16*>(smem);
    TIN* ts = reinterpret_cast<TIN*>(smem + al16((size_t)WN * 2));
    const int tid = threadIdx.x;
    for (int e = tid; e < WN / 8; e += C3_THREADS)
        reinterpret_cast<uint4*>(ws)[e] = reinterpret_cast<const uint4*>(w)[e];
    load_box<CIN>(v, in, ts, blockIdx.x * C3_X - 1, blockIdx.y * C3_Y - 1, blockIdx.z * C3_P - 1, C3_HX, C3_HY, C3_HZ,
                  tid, C3_THREADS);
    __syncthreads();
    const int tx = tid % C3_X, ty = tid / C3_X;
    float acc[C3_P][COUT];
#pragma unroll
    for (int q = 0; q < C3_P; ++q)
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[q][co] = BWD ? 0.f : bias[co];
    constexpr int CC = CIN % 4 == 0 ? 4 : 2;
    constexpr int ZS = C3_HX * C3_HY * CIN;
#pragma unroll 1
    for (int dy = 0; dy < 3; ++dy) {
#pragma unroll 1
        for (int dx = 0; dx < 3; ++dx) {
            const TIN* colp = ts + ((ty + dy) * C3_HX + tx + dx) * CIN;
#pragma unroll 1
            for (int c0 = 0; c0 < CIN; c0 += CC) {
                float col[C3_P + 2][CC];
#pragma unroll
                for (int t = 0; t < C3_P + 2; ++t) ldc<CC>(colp + t * ZS + c0, col[t]);
#pragma unroll
                for (int dz = 0; dz < 3; ++dz) {
                    const bf16* wr = ws + (((dz * 3 + dy) * 3 + dx) * CIN + c0) * COUT;
#pragma unroll
                    for (int c = 0; c < CC; ++c) {
                        float wv[COUT];
                        ldrow<COUT>(wr + c * COUT, wv);
#pragma unroll
                        for (int q = 0; q < C3_P; ++q)
#pragma unroll
                            for (int co = 0; co < COUT; ++co) acc[q][co] = fmaf(col[q + dz][c], wv[co], acc[q][co]);
                    }
                }
            }
        }
    }
    const int gx = blockIdx.x * C3_X + tx, gy = blockIdx.y * C3_Y + ty;
    if (gx >= v.nx || gy >= v.ny) return;
#pragma unroll
    for (int q = 0; q < C3_P; ++q) {
        const int gz = blockIdx.z * C3_P + q;
        if (gz < v.nz) {
            const long long p = ((long long)gz * v.ny + gy) * v.nx + gx;
            if constexpr (!BWD) {
                float a[COUT];
#pragma unroll
                for (int co = 0; co < COUT; ++co) a[co] = silu(acc[q][co]);
                strow<COUT>(zout + p * COUT, acc[q]);
                strow<COUT>(aout + p * COUT, a);
            } else {
                float zp[COUT];
                ldrow<COUT>(zprev + p * COUT, zp);
#pragma unroll
                for (int co = 0; co < COUT; ++co) {
                    const float g = acc[q][co] + (extra ? extra[p * COUT + co] : 0.f);
                    gout[p * COUT + co] = g * dsilu(zp[co]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------- tensor-core 3x3x3 ----
// Forward convolution as an implicit GEMM on the 5th-generation tensor cores: per block a
// 128-point tile (16 x 8 x 1) of outputs, D[point][cout] = sum over 27 taps and CIN channels
// of in[point + tap][ci] w[tap][ci][co], BF16 operands (tcgen05.mma kind::f16, A and B both
// BF16), FP32 accumulator in TMEM.  The halo tile (18 x 10 x 3 points) is staged once; for
// each group of taps the shifted input rows are copied into the canonical K-major,
// no-swizzle layout (core matrix = 8 rows x 16 bytes) and one thread issues CIN/16 MMAs per
// tap.  Weights for all taps are staged once per block in the same layout.  Every mbarrier
// wait is bounded; a block that gives up flags the error, drains its MMAs and frees TMEM.
constexpr int TCC_THREADS = 256;
constexpr int TCC_X = 16, TCC_Y = 8, TCC_M = 128;
constexpr int TCC_HX = TCC_X + 2, TCC_HY = TCC_Y + 2, TCC_HZ = 3;
constexpr long long TCC_SPIN_LIMIT = 1LL << 22;

__device__ __forceinline__ uint32_t tcc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool tcc_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = tcc_smem(bar);
    for (long long i = 0; i < TCC_SPIN_LIMIT; ++i) {
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

__device__ __forceinline__ uint64_t tcc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100; no swizzle, base offset 0
    return d;
}

// D = F32, A = B = BF16, both K-major, M = 128
__host__ __device__ constexpr uint32_t tcc_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TCC_M >> 4) << 24);
}

// byte offset of element (row, k) in an R-row canonical K-major bf16 tile
__device__ __forceinline__ int tcc_off(int row, int k, int R) {
    return (((k >> 3) * (R >> 3) + (row >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1);
}

template <int CIN, int COUT>
constexpr int tcc_group() { return CIN == 16 ? 27 : 9; }  // taps staged per MMA batch

template <int CIN, int COUT>
constexpr size_t tcc_smem_bytes() {
    return (size_t)27 * COUT * CIN * 2                              // weights
           + (size_t)tcc_group<CIN, COUT>() * TCC_M * CIN * 2       // A rows for a group of taps
           + al16((size_t)TCC_HX * TCC_HY * TCC_HZ * CIN * 2);      // halo
}

// BWD = true: data gradient of a convolution (w = flipped, transposed weights, in = the
// output gradient rounded to BF16): g = sum * silu'(zprev), stored in FP32 to gout.
template <int CIN, int COUT, bool BWD>
__global__ void __launch_bounds__(TCC_THREADS, 1)
    conv3_tc_kernel(Vol v, const bf16* __restrict__ in, const bf16* __restrict__ w, const float* __restrict__ bias,
                    bf16* __restrict__ zout, bf16* __restrict__ aout, float* __restrict__ gout,
                    const bf16* __restrict__ zprev, int* __restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t bar;
    constexpr int G = tcc_group<CIN, COUT>();
    constexpr int W_BYTES = 27 * COUT * CIN * 2, A_TAP = TCC_M * CIN * 2;
    constexpr int NCOL = COUT < 32 ? 32 : COUT;  // TMEM columns (power of two >= 32)
    unsigned char* wsm = smem;
    unsigned char* asm_ = smem + W_BYTES;
    bf16* halo = reinterpret_cast<bf16*>(smem + W_BYTES + G * A_TAP);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tcc_smem(&s_tmem)),
                     "r"(NCOL));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tcc_smem(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights: tap t, element (co, ci) of the N x K operand
    for (int e = tid; e < 27 * CIN * COUT; e += TCC_THREADS) {
        const int co = e % COUT, ci = (e / COUT) % CIN, t = e / (COUT * CIN);
        *reinterpret_cast<bf16*>(wsm + t * COUT * CIN * 2 + tcc_off(co, ci, COUT)) = w[e];
    }
    const int x0 = blockIdx.x * TCC_X, y0 = blockIdx.y * TCC_Y, z0 = blockIdx.z;
    load_box<CIN>(v, in, halo, x0 - 1, y0 - 1, z0 - 1, TCC_HX, TCC_HY, TCC_HZ, tid, TCC_THREADS);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    constexpr uint32_t lbo_a = (TCC_M / 8) * 128, lbo_b = (COUT / 8) * 128, sbo = 128;
    constexpr uint32_t idesc = tcc_idesc(COUT);
    bool ok = true;
    uint32_t phase = 0;
    for (int t0 = 0; t0 < 27; t0 += G) {
        if (t0 > 0) {  // the previous group's MMAs read the A buffers: wait before rewriting them
            if (!tcc_wait(&bar, phase)) ok = false;
            phase ^= 1;
        }
        if (!__syncthreads_and(ok)) break;
        // A rows: for tap t0 + g, row m = output point (m % 16, m / 16), 16-byte chunks of 8 channels
        constexpr int CH = CIN / 8;
        for (int e = tid; e < G * TCC_M * CH; e += TCC_THREADS) {
            const int c = e % CH, m = (e / CH) % TCC_M, gi = e / (CH * TCC_M);
            const int t = t0 + gi, tz = t / 9, ty = (t / 3) % 3, tx = t % 3;
            const int hx = (m % TCC_X) + tx, hy = (m / TCC_X) + ty;
            const uint4 val = *reinterpret_cast<const uint4*>(halo + ((tz * TCC_HY + hy) * TCC_HX + hx) * CIN + c * 8);
            *reinterpret_cast<uint4*>(asm_ + gi * A_TAP + (((c * (TCC_M / 8) + (m >> 3)) << 7) + ((m & 7) << 4))) = val;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            for (int gi = 0; gi < G; ++gi) {
                const uint32_t a0 = tcc_smem(asm_ + gi * A_TAP), b0 = tcc_smem(wsm + (t0 + gi) * COUT * CIN * 2);
#pragma unroll
                for (int kk = 0; kk < CIN / 16; ++kk) {
                    const uint64_t da = tcc_desc(a0 + kk * 2 * lbo_a, lbo_a, sbo);
                    const uint64_t db = tcc_desc(b0 + kk * 2 * lbo_b, lbo_b, sbo);
                    const uint32_t acc = (t0 == 0 && gi == 0 && kk == 0) ? 0u : 1u;
                    const uint32_t zero = 0;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                        ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(zero));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             tcc_smem(&bar))
                         : "memory");
        }
    }
    // the last group (or a group cut short by an error) still has MMAs in flight
    if (!tcc_wait(&bar, phase)) ok = false;
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0) atomicExch(error, 1);
    } else {
        // lane = output point; warps w and w + 4 split the output channels
        const int q4 = warp & 3, half = warp >> 2;
        const int m = q4 * 32 + lane;
        const int gx = x0 + (m % TCC_X), gy = y0 + (m / TCC_X);
        constexpr int HC = COUT / 2;
        float z[HC];
#pragma unroll
        for (int c0 = 0; c0 < HC; c0 += 8) {
            uint32_t r[8];
            const uint32_t addr = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)(half * HC + c0);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 8; ++q) z[c0 + q] = __uint_as_float(r[q]) + (BWD ? 0.f : bias[half * HC + c0 + q]);
        }
        if (gx < v.nx && gy < v.ny) {
            const long long p = ((long long)z0 * v.ny + gy) * v.nx + gx;
            if constexpr (BWD) {
                float zp[HC];
                ldrow<HC>(zprev + p * COUT + half * HC, zp);
#pragma unroll
                for (int c = 0; c < HC; ++c) gout[p * COUT + half * HC + c] = z[c] * dsilu(zp[c]);
            } else {
                float a[HC];
#pragma unroll
                for (int c = 0; c < HC; ++c) a[c] = silu(z[c]);
                strow<HC>(zout + p * COUT + half * HC, z);
                strow<HC>(aout + p * COUT + half * HC, a);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL));
}

// wT[tap][co][ci] = w[26 - tap][ci][co]: the data gradient of a 3x3x3 convolution is the
// convolution of the output gradient with the flipped, transposed kernel.
__global__ void conv3_flip_kernel(int cin, int cout, const bf16* __restrict__ w, bf16* __restrict__ wT) {
    const int n = 27 * cin * cout;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const int ci = e % cin, co = (e / cin) % cout, tap = e / (cin * cout);
        wT[e] = w[((26 - tap) * cin + ci) * cout + co];
    }
}

// Weight and bias gradients of a 3x3x3 convolution: dw[tap][ci][co] += sum_p in[p+off][ci] dz[p][co].
// Each thread owns one (tap, channel pair) item and all output channels; blocks loop over
// tiles and add their partial sums once at the end.
constexpr int WG_THREADS = 256;
template <int CIN, int COUT>
constexpr size_t wgrad_smem() {
    return al16((size_t)C3_HPTS * CIN * 2) + (size_t)C3_X * C3_Y * C3_P * COUT * 4;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(WG_THREADS) conv3_wgrad_kernel(Vol v, const bf16* __restrict__ in,
                                                                 const float* __restrict__ dz, float* __restrict__ dw,
                                                                 float* __restrict__ db) {
    extern __shared__ __align__(16) unsigned char smem[];
    bf16* ts = reinterpret_cast<bf16*>(smem);
    float* ds = reinterpret_cast<float*>(smem + al16((size_t)C3_HPTS * CIN * 2));
    constexpr int CP = CIN / 2, NI = 27 * CP, IPT = (NI + WG_THREADS - 1) / WG_THREADS;
    constexpr int TP = C3_X * C3_Y * C3_P;
    const int tid = threadIdx.x;
    int hoff[IPT];
    bool act[IPT];
#pragma unroll
    for (int it = 0; it < IPT; ++it) {
        const int item = tid + it * WG_THREADS;
        act[it] = item < NI;
        const int tap = act[it] ? item / CP : 0, cp = act[it] ? item % CP : 0;
        const int tz = tap / 9, ty = (tap / 3) % 3, tx = tap % 3;
        hoff[it] = ((tz * C3_HY + ty) * C3_HX + tx) * CIN + 2 * cp;
    }
    float acc[IPT][2][COUT];
#pragma unroll
    for (int it = 0; it < IPT; ++it)
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[it][0][co] = acc[it][1][co] = 0.f;
    float bacc = 0.f;
    const int tbx = (v.nx + C3_X - 1) / C3_X, tby = (v.ny + C3_Y - 1) / C3_Y, tbz = (v.nz + C3_P - 1) / C3_P;
    const int total = tbx * tby * tbz;
    for (int tile = blockIdx.x; tile < total; tile += gridDim.x) {
        const int bx = tile % tbx, by = (tile / tbx) % tby, bz = tile / (tbx * tby);
        __syncthreads();
        load_box<CIN>(v, in, ts, bx * C3_X - 1, by * C3_Y - 1, bz * C3_P - 1, C3_HX, C3_HY, C3_HZ, tid, WG_THREADS);
        load_box<COUT>(v, dz, ds, bx * C3_X, by * C3_Y, bz * C3_P, C3_X, C3_Y, C3_P, tid, WG_THREADS);
        __syncthreads();
#pragma unroll 1
        for (int q = 0; q < TP; ++q) {
            const int lx = q % C3_X, ly = (q / C3_X) % C3_Y, lz = q / (C3_X * C3_Y);
            const int base = ((lz * C3_HY + ly) * C3_HX + lx) * CIN;
            float g[COUT];
            ldrow<COUT>(ds + q * COUT, g);
            if (tid < COUT) bacc += ds[q * COUT + tid];
#pragma unroll
            for (int it = 0; it < IPT; ++it) {
                if (act[it]) {
                    float a[2];
                    ldc<2>(ts + base + hoff[it], a);
#pragma unroll
                    for (int co = 0; co < COUT; ++co) {
                        acc[it][0][co] = fmaf(a[0], g[co], acc[it][0][co]);
                        acc[it][1][co] = fmaf(a[1], g[co], acc[it][1][co]);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int it = 0; it < IPT; ++it) {
        if (!act[it]) continue;
        const int item = tid + it * WG_THREADS, tap = item / CP, cp = item % CP;
        float* d0 = dw + ((size_t)tap * CIN + 2 * cp) * COUT;
#pragma unroll
        for (int co = 0; co < COUT; ++co) {
            atomicAdd(d0 + co, acc[it][0][co]);
            atomicAdd(d0 + COUT + co, acc[it][1][co]);
        }
    }
    if (tid < COUT) atomicAdd(db + tid, bacc);
}

// ---------------------------------------------------------------- down / up ----------
// child t of coarse point (X, Y, Z): (2X + (t&1), 2Y + ((t>>1)&1), 2Z + (t>>2))
__device__ __forceinline__ void decode(const Vol v, long long p, int& x, int& y, int& z) {
    x = (int)(p % v.nx);
    y = (int)((p / v.nx) % v.ny);
    z = (int)(p / ((long long)v.nx * v.ny));
}
__device__ __forceinline__ long long lin(const Vol v, int x, int y, int z) {
    return ((long long)z * v.ny + y) * v.nx + x;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(256) down_fwd_kernel(Vol f, Vol c, const bf16* __restrict__ in,
                                                       const bf16* __restrict__ w, const float* __restrict__ bias,
                                                       bf16* __restrict__ zout, bf16* __restrict__ aout) {
    __shared__ __align__(16) bf16 ws[8 * CIN * COUT];
    for (int e = threadIdx.x; e < 8 * CIN * COUT / 8; e += blockDim.x)
        reinterpret_cast<uint4*>(ws)[e] = reinterpret_cast<const uint4*>(w)[e];
    __syncthreads();
    for (long long P = (long long)blockIdx.x * blockDim.x + threadIdx.x; P < c.n(); P += (long long)gridDim.x * blockDim.x) {
        int X, Y, Z;
        decode(c, P, X, Y, Z);
        float acc[COUT];
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] = bias[co];
#pragma unroll 1
        for (int t = 0; t < 8; ++t) {
            const int fx = 2 * X + (t & 1), fy = 2 * Y + ((t >> 1) & 1), fz = 2 * Z + (t >> 2);
            if (fx >= f.nx || fy >= f.ny || fz >= f.nz) continue;
            const bf16* ip = in + lin(f, fx, fy, fz) * CIN;
#pragma unroll 1
            for (int c0 = 0; c0 < CIN; c0 += 4) {
                float x4[4];
                ldc<4>(ip + c0, x4);
#pragma unroll
                for (int cc = 0; cc < 4; ++cc) {
                    float wv[COUT];
                    ldrow<COUT>(ws + (t * CIN + c0 + cc) * COUT, wv);
#pragma unroll
                    for (int co = 0; co < COUT; ++co) acc[co] = fmaf(x4[cc], wv[co], acc[co]);
                }
            }
        }
        float a[COUT];
#pragma unroll
        for (int co = 0; co < COUT; ++co) a[co] = silu(acc[co]);
        strow<COUT>(zout + P * COUT, acc);
        strow<COUT>(aout + P * COUT, a);
    }
}

// data gradient of down: g[p][ci] = (sum_co w[t(p)][ci][co] dz[P(p)][co] + extra[p][ci]) * silu'(zprev[p][ci])
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) down_bwd_kernel(Vol f, Vol c, const float* __restrict__ dzc,
                                                       const bf16* __restrict__ w, const float* __restrict__ extra,
                                                       const bf16* __restrict__ zprev, float* __restrict__ gout) {
    __shared__ __align__(16) bf16 ws[8 * CIN * COUT];
    for (int e = threadIdx.x; e < 8 * CIN * COUT / 8; e += blockDim.x)
        reinterpret_cast<uint4*>(ws)[e] = reinterpret_cast<const uint4*>(w)[e];
    __syncthreads();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < f.n(); p += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(f, p, x, y, z);
        const int t = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2);
        float g[COUT];
        ldrow<COUT>(dzc + lin(c, x >> 1, y >> 1, z >> 1) * COUT, g);
        float zp[CIN];
        ldrow<CIN>(zprev + p * CIN, zp);
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) {
            float wv[COUT];
            ldrow<COUT>(ws + (t * CIN + ci) * COUT, wv);
            float s = 0.f;
#pragma unroll
            for (int co = 0; co < COUT; ++co) s = fmaf(wv[co], g[co], s);
            if (extra) s += extra[p * CIN + ci];
            gout[p * CIN + ci] = s * dsilu(zp[ci]);
        }
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(256) up_fwd_kernel(Vol f, Vol c, const bf16* __restrict__ in,
                                                     const bf16* __restrict__ w, const float* __restrict__ bias,
                                                     const bf16* __restrict__ skip, bf16* __restrict__ zout,
                                                     bf16* __restrict__ aout) {
    __shared__ __align__(16) bf16 ws[8 * CIN * COUT];
    for (int e = threadIdx.x; e < 8 * CIN * COUT / 8; e += blockDim.x)
        reinterpret_cast<uint4*>(ws)[e] = reinterpret_cast<const uint4*>(w)[e];
    __syncthreads();
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < f.n(); p += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(f, p, x, y, z);
        const int t = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2);
        float acc[COUT];
        ldrow<COUT>(skip + p * COUT, acc);
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] += bias[co];
        const bf16* ip = in + lin(c, x >> 1, y >> 1, z >> 1) * CIN;
#pragma unroll 1
        for (int c0 = 0; c0 < CIN; c0 += 4) {
            float x4[4];
            ldc<4>(ip + c0, x4);
#pragma unroll
            for (int cc = 0; cc < 4; ++cc) {
                float wv[COUT];
                ldrow<COUT>(ws + (t * CIN + c0 + cc) * COUT, wv);
#pragma unroll
                for (int co = 0; co < COUT; ++co) acc[co] = fmaf(x4[cc], wv[co], acc[co]);
            }
        }
        float a[COUT];
#pragma unroll
        for (int co = 0; co < COUT; ++co) a[co] = silu(acc[co]);
        strow<COUT>(zout + p * COUT, acc);
        strow<COUT>(aout + p * COUT, a);
    }
}

// data gradient of up: g[P][ci] = sum_t sum_co w[t][ci][co] dz[child(P,t)][co] * silu'(zprev[P][ci])
template <int CIN, int COUT>
__global__ void __launch_bounds__(256) up_bwd_kernel(Vol f, Vol c, const float* __restrict__ dzf,
                                                     const bf16* __restrict__ w, const bf16* __restrict__ zprev,
                                                     float* __restrict__ gout) {
    __shared__ __align__(16) bf16 ws[8 * CIN * COUT];
    for (int e = threadIdx.x; e < 8 * CIN * COUT / 8; e += blockDim.x)
        reinterpret_cast<uint4*>(ws)[e] = reinterpret_cast<const uint4*>(w)[e];
    __syncthreads();
    for (long long P = (long long)blockIdx.x * blockDim.x + threadIdx.x; P < c.n(); P += (long long)gridDim.x * blockDim.x) {
        int X, Y, Z;
        decode(c, P, X, Y, Z);
        float acc[CIN];
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.f;
#pragma unroll 1
        for (int t = 0; t < 8; ++t) {
            const int fx = 2 * X + (t & 1), fy = 2 * Y + ((t >> 1) & 1), fz = 2 * Z + (t >> 2);
            if (fx >= f.nx || fy >= f.ny || fz >= f.nz) continue;
            float g[COUT];
            ldrow<COUT>(dzf + lin(f, fx, fy, fz) * COUT, g);
#pragma unroll
            for (int ci = 0; ci < CIN; ++ci) {
                float wv[COUT];
                ldrow<COUT>(ws + (t * CIN + ci) * COUT, wv);
#pragma unroll
                for (int co = 0; co < COUT; ++co) acc[ci] = fmaf(wv[co], g[co], acc[ci]);
            }
        }
        float zp[CIN];
        ldrow<CIN>(zprev + P * CIN, zp);
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) gout[P * CIN + ci] = acc[ci] * dsilu(zp[ci]);
    }
}

// Weight/bias gradients of down (UP = false: pairs in[child(P,t)], dz[P]) and up
// (UP = true: pairs in[P], dz[child(P,t)]).  Thread = (t, ci) item with COUT accumulators.
template <int CIN, int COUT, bool UP>
__global__ void __launch_bounds__(256) pair_wgrad_kernel(Vol f, Vol c, const bf16* __restrict__ in,
                                                         const float* __restrict__ dz, float* __restrict__ dw,
                                                         float* __restrict__ db) {
    constexpr int CPB = 16;
    static_assert(8 * CIN <= 256, "one (t, ci) item per thread");
    __shared__ __align__(16) float as[CPB][8][CIN];
    __shared__ __align__(16) float gs[CPB][8][COUT];
    const int tid = threadIdx.x;
    const bool act = tid < 8 * CIN;
    const int t = tid / CIN, ci = tid % CIN;
    float acc[COUT];
#pragma unroll
    for (int co = 0; co < COUT; ++co) acc[co] = 0.f;
    float bacc = 0.f;
    const long long nc = c.n();
    for (long long base = (long long)blockIdx.x * CPB; base < nc; base += (long long)gridDim.x * CPB) {
        __syncthreads();
        for (int e = tid; e < CPB * 8 * CIN; e += 256) {
            const int pc = e / (8 * CIN), r = e % (8 * CIN), tt = r / CIN, cc = r % CIN;
            const long long P = base + pc;
            float val = 0.f;
            if (P < nc) {
                int X, Y, Z;
                decode(c, P, X, Y, Z);
                const int fx = 2 * X + (tt & 1), fy = 2 * Y + ((tt >> 1) & 1), fz = 2 * Z + (tt >> 2);
                if (UP) val = __bfloat162float(in[P * CIN + cc]);
                else if (fx < f.nx && fy < f.ny && fz < f.nz) val = __bfloat162float(in[lin(f, fx, fy, fz) * CIN + cc]);
            }
            as[pc][tt][cc] = val;
        }
        for (int e = tid; e < CPB * 8 * COUT; e += 256) {
            const int pc = e / (8 * COUT), r = e % (8 * COUT), tt = r / COUT, cc = r % COUT;
            const long long P = base + pc;
            float val = 0.f;
            if (P < nc) {
                int X, Y, Z;
                decode(c, P, X, Y, Z);
                const int fx = 2 * X + (tt & 1), fy = 2 * Y + ((tt >> 1) & 1), fz = 2 * Z + (tt >> 2);
                if (!UP) val = dz[P * COUT + cc];
                else if (fx < f.nx && fy < f.ny && fz < f.nz) val = dz[lin(f, fx, fy, fz) * COUT + cc];
            }
            gs[pc][tt][cc] = val;
        }
        __syncthreads();
        if (act) {
#pragma unroll 1
            for (int pc = 0; pc < CPB; ++pc) {
                const float a = as[pc][t][ci];
#pragma unroll
                for (int co = 0; co < COUT; ++co) acc[co] = fmaf(a, gs[pc][t][co], acc[co]);
            }
        }
        if (tid < COUT) {
            for (int pc = 0; pc < CPB; ++pc) {
                if (UP)
                    for (int tt = 0; tt < 8; ++tt) bacc += gs[pc][tt][tid];
                else
                    bacc += gs[pc][0][tid];
            }
        }
    }
    if (act)
        for (int co = 0; co < COUT; ++co) atomicAdd(dw + ((size_t)t * CIN + ci) * COUT + co, acc[co]);
    if (tid < COUT) atomicAdd(db + tid, bacc);
}

// ---------------------------------------------------------------- head + loss ----------
template <int C>
__global__ void __launch_bounds__(256) head_fwd_kernel(long long n, const bf16* __restrict__ a,
                                                       const bf16* __restrict__ w, const float* __restrict__ bias,
                                                       float* __restrict__ y) {
    float wv[C];
    ldrow<C>(w, wv);
    const float b = bias[0];
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        float av[C];
        ldrow<C>(a + p * C, av);
        float s = b;
#pragma unroll
        for (int c = 0; c < C; ++c) s = fmaf(wv[c], av[c], s);
        y[p] = s;
    }
}

// Backward through the head: given dL/dy, writes dz of the last hidden layer and adds the
// head's weight/bias gradients to dw / db.
template <int C>
__global__ void __launch_bounds__(256) head_bwd_kernel(long long n, const float* __restrict__ dy,
                                                       const bf16* __restrict__ a, const bf16* __restrict__ z,
                                                       const bf16* __restrict__ w, float* __restrict__ dzout,
                                                       float* __restrict__ dw, float* __restrict__ db) {
    float wv[C];
    ldrow<C>(w, wv);
    float gw[C];
#pragma unroll
    for (int c = 0; c < C; ++c) gw[c] = 0.f;
    float gb = 0.f;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const float gy = dy[p];
        float av[C], zv[C];
        ldrow<C>(a + p * C, av);
        ldrow<C>(z + p * C, zv);
#pragma unroll
        for (int c = 0; c < C; ++c) {
            gw[c] = fmaf(av[c], gy, gw[c]);
            dzout[p * C + c] = wv[c] * gy * dsilu(zv[c]);
        }
        gb += gy;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gb += __shfl_xor_sync(0xffffffffu, gb, o);
#pragma unroll
        for (int c = 0; c < C; ++c) gw[c] += __shfl_xor_sync(0xffffffffu, gw[c], o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(db, gb);
#pragma unroll
        for (int c = 0; c < C; ++c) atomicAdd(dw + c, gw[c]);
    }
}

// ---------------------------------------------------------------- loss ----------------
// e = y - t on interior points (y may be null: a zero correction), 0 on faces
__global__ void err_init_kernel(Vol v, const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ e) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < v.n(); p += (long long)gridDim.x * blockDim.x) {
        int x, yy, zz;
        decode(v, p, x, yy, zz);
        const bool interior = x > 0 && x + 1 < v.nx && yy > 0 && yy + 1 < v.ny && zz > 0 && zz + 1 < v.nz;
        e[p] = interior ? (y ? y[p] : 0.f) - t[p] : 0.f;
    }
}

// One Jacobi sweep on an error field (zero source, zero faces): out = J in.  J is symmetric,
// so it is also its own adjoint in the gradient.
__global__ void err_jacobi_kernel(Vol v, float cx, float cy, float cz, float iden, const float* __restrict__ in,
                                  float* __restrict__ out) {
    const long long sxy = (long long)v.nx * v.ny;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < v.n(); p += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        decode(v, p, x, y, z);
        const bool interior = x > 0 && x + 1 < v.nx && y > 0 && y + 1 < v.ny && z > 0 && z + 1 < v.nz;
        out[p] = interior ? (cx * (in[p - 1] + in[p + 1]) + cy * (in[p - v.nx] + in[p + v.nx]) +
                             cz * (in[p - sxy] + in[p + sxy])) * iden
                          : 0.f;
    }
}

// red += scale * sum e^2; g = c * e (g may alias nothing)
__global__ void sq_sum_kernel(long long n, const float* __restrict__ e, double scale, double* __restrict__ red,
                              float* __restrict__ g, float c) {
    double l = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const float v = e[p];
        l += (double)v * v;
        if (g) g[p] = c * v;
    }
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0) atomicAdd(red, l * scale);
}

// dy = a * e0 + b
__global__ void axpy_kernel(long long n, float a, const float* __restrict__ e0, const float* __restrict__ b,
                            float* __restrict__ dy) {
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        dy[p] = a * e0[p] + (b ? b[p] : 0.f);
}

// ---------------------------------------------------------------- optimiser ----------
__global__ void adam_kernel(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, bf16* __restrict__ pb, float lr, float b1, float b2, float eps,
                            float c1, float c2, float gscale) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i] * gscale;
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] = pi;
        pb[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void to_bf16_kernel(long long n, const float* __restrict__ p, bf16* __restrict__ pb) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        pb[i] = __float2bfloat16_rn(p[i]);
}

// network input: [4 pi hbar^2 rho / s, vup / s] in BF16
__global__ void build_input_kernel(long long n, const double* __restrict__ rho, const double* __restrict__ vup,
                                   const double* __restrict__ s, double h2, bf16* __restrict__ x) {
    const double is = 1.0 / *s;
    const double c = 4.0 * 3.14159265358979323846 * h2 * is;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        reinterpret_cast<uint32_t*>(x)[p] = pack_bf2((float)(c * rho[p]), (float)(vup[p] * is));
    }
}

// ---- learned Davidson preconditioner: t = t0 + s * net([c r / s, t0 / s]), s = max|t0| ------
__global__ void absmax_kernel(long long n, const double* __restrict__ x, unsigned long long* __restrict__ out) {
    double m = 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[p]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
__global__ void pc_input_kernel(long long n, const double* __restrict__ r, const double* __restrict__ t0,
                                const unsigned long long* __restrict__ sbits, double c, bf16* __restrict__ x) {
    const double s = __longlong_as_double((long long)*sbits);
    const double is = s > 0.0 ? 1.0 / s : 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        reinterpret_cast<uint32_t*>(x)[p] = pack_bf2((float)(c * r[p] * is), (float)(t0[p] * is));
}
// interior points: t += s y
__global__ void pc_apply_kernel(Grid g, const float* __restrict__ y, const unsigned long long* __restrict__ sbits,
                                double* __restrict__ t) {
    const double s = __longlong_as_double((long long)*sbits);
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const bool face = i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz;
        if (!face) t[p] += s * (double)y[p];
    }
}
// training target (t* - t0) / s on the interior, 0 on faces
__global__ void pc_target_kernel(Grid g, const double* __restrict__ ts, const double* __restrict__ t0,
                                 const unsigned long long* __restrict__ sbits, float* __restrict__ t) {
    const double s = __longlong_as_double((long long)*sbits);
    const double is = s > 0.0 ? 1.0 / s : 0.0;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const bool face = i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz;
        t[p] = face ? 0.f : (float)((ts[p] - t0[p]) * is);
    }
}

// training target: (v - vup) / s on the interior, 0 on faces
__global__ void build_target_kernel(Grid g, const double* __restrict__ v, const double* __restrict__ vup,
                                    const double* __restrict__ s, float* __restrict__ t) {
    const double is = 1.0 / *s;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const bool face = i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz;
        t[p] = face ? 0.f : (float)((v[p] - vup[p]) * is);
    }
}

// out = vup + s * y on the interior
__global__ void combine_kernel(Grid g, const double* __restrict__ vup, const float* __restrict__ y,
                               const double* __restrict__ s, double* __restrict__ out) {
    const double sc = *s;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.N; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p % g.nx), j = (int)((p / g.nx) % g.ny), k = (int)(p / ((long long)g.nx * g.ny));
        const bool face = i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz;
        out[p] = face ? 0.0 : vup[p] + sc * (double)y[p];
    }
}

inline int blocks_for(dft_context* ctx, long long n, int per = 256) {
    const long long b = (n + per - 1) / per;
    return (int)std::max<long long>(1, std::min<long long>(b, (long long)ctx->num_sms * 8));
}

template <typename T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    T* get(size_t want) {
        if (want > n) {
            if (p) cudaFree(p);
            p = nullptr;
            n = 0;
            DFT_CUDA(cudaMalloc(&p, std::max<size_t>(want, 1) * sizeof(T)));
            n = want;
        }
        return p;
    }
};

enum LayerType { L_CONV3 = 0, L_DOWN = 1, L_UP = 2, L_HEAD = 3 };
struct Layer {
    int type, cin, cout, level;
    size_t w, b;  // offsets into the parameter vector (w a multiple of 8)
    size_t taps() const { return type == L_CONV3 ? 27 : (type == L_HEAD ? 1 : 8); }
};

}  // namespace
}  // namespace dftb

struct dft_pnet {
    dft_context* ctx = nullptr;
    int in_ch = 2;
    std::vector<dftb::Layer> L;
    size_t np = 0;
    dftb::DBuf<float> p, g, m, v;
    dftb::DBuf<__nv_bfloat16> pb;
    long step = 0;
    // activations (z, a per layer), gradients, scratch
    dftb::DBuf<__nv_bfloat16> x, z[12], a[12], wT;
    dftb::DBuf<float> y, dz[12], t, e0, e1, e2, dy;
    dftb::DBuf<double> red;
    dftb::DBuf<int> tc_err;  // set by a tensor-core convolution block whose wait timed out
    dftb::DBuf<__nv_bfloat16> dzb;  // output gradient rounded to BF16 for the tensor-core data gradient
    dftb::DBuf<unsigned long long> sbits;  // per-band scale of the preconditioner's input/output
};

namespace dftb {
namespace {

using PNet = dft_pnet;

template <typename K>
void set_smem(K kern, size_t bytes) {
    if (bytes > 48 * 1024) DFT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

template <int CIN, int COUT, typename TIN, bool BWD>
void launch_conv3(dft_context* ctx, Vol v, const TIN* in, const bf16* w, const float* bias, bf16* z, bf16* a,
                  float* g, const float* extra, const bf16* zprev) {
    constexpr size_t sm = conv3_smem<CIN, COUT, TIN>();
    static bool once = false;
    if (!once) {
        set_smem(conv3_kernel<CIN, COUT, TIN, BWD>, sm);
        once = true;
    }
    dim3 grid((v.nx + C3_X - 1) / C3_X, (v.ny + C3_Y - 1) / C3_Y, (v.nz + C3_P - 1) / C3_P);
    conv3_kernel<CIN, COUT, TIN, BWD><<<grid, C3_THREADS, sm, ctx->stream>>>(v, in, w, bias, z, a, g, extra, zprev);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

template <int CIN, int COUT>
void launch_conv3_tc(dft_context* ctx, Vol v, const bf16* in, const bf16* w, const float* bias, bf16* z, bf16* a,
                     int* err) {
    constexpr size_t sm = tcc_smem_bytes<CIN, COUT>();
    static bool once = false;
    if (!once) {
        set_smem(conv3_tc_kernel<CIN, COUT, false>, sm);
        once = true;
    }
    dim3 grid((v.nx + TCC_X - 1) / TCC_X, (v.ny + TCC_Y - 1) / TCC_Y, v.nz);
    conv3_tc_kernel<CIN, COUT, false><<<grid, TCC_THREADS, sm, ctx->stream>>>(v, in, w, bias, z, a, nullptr, nullptr,
                                                                              err);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

// Data gradient on the tensor cores: the output gradient dz (FP32) is rounded to BF16, then
// convolved with the flipped, transposed weights wT; gout = result * silu'(zprev).
template <int C>
void launch_conv3_tc_bwd(dft_context* ctx, PNet* n, Vol v, const float* dz, const bf16* wT, float* gout,
                         const bf16* zprev, int* err) {
    constexpr size_t sm = tcc_smem_bytes<C, C>();
    static bool once = false;
    if (!once) {
        set_smem(conv3_tc_kernel<C, C, true>, sm);
        once = true;
    }
    const long long cnt = v.n() * C;
    bf16* dzb = n->dzb.get((size_t)cnt);
    to_bf16_kernel<<<blocks_for(ctx, cnt), 256, 0, ctx->stream>>>(cnt, dz, dzb);
    dim3 grid((v.nx + TCC_X - 1) / TCC_X, (v.ny + TCC_Y - 1) / TCC_Y, v.nz);
    conv3_tc_kernel<C, C, true><<<grid, TCC_THREADS, sm, ctx->stream>>>(v, dzb, wT, nullptr, nullptr, nullptr, gout,
                                                                       zprev, err);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
}

template <int CIN, int COUT>
void launch_wgrad(dft_context* ctx, Vol v, const bf16* in, const float* dz, float* dw, float* db) {
    constexpr size_t sm = wgrad_smem<CIN, COUT>();
    static bool once = false;
    if (!once) {
        set_smem(conv3_wgrad_kernel<CIN, COUT>, sm);
        once = true;
    }
    const long long tiles = (long long)((v.nx + C3_X - 1) / C3_X) * ((v.ny + C3_Y - 1) / C3_Y) * ((v.nz + C3_P - 1) / C3_P);
    const int nb = (int)std::min<long long>(tiles, 2LL * ctx->num_sms);
    conv3_wgrad_kernel<CIN, COUT><<<nb, WG_THREADS, sm, ctx->stream>>>(v, in, dz, dw, db);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void flip(dft_context* ctx, int cin, int cout, const bf16* w, bf16* wT) {
    conv3_flip_kernel<<<blocks_for(ctx, 27LL * cin * cout), 256, 0, ctx->stream>>>(cin, cout, w, wT);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void build_layers(PNet* n) {
    const int C0 = 16, C1 = 32, C2 = 32;
    struct D {
        int type, cin, cout, level;
    };
    const D d[12] = {{L_CONV3, n->in_ch, C0, 0}, {L_CONV3, C0, C0, 0}, {L_DOWN, C0, C1, 1},  {L_CONV3, C1, C1, 1},
                     {L_DOWN, C1, C2, 2},        {L_CONV3, C2, C2, 2}, {L_CONV3, C2, C2, 2}, {L_UP, C2, C1, 1},
                     {L_CONV3, C1, C1, 1},       {L_UP, C1, C0, 0},    {L_CONV3, C0, C0, 0}, {L_HEAD, C0, 1, 0}};
    size_t off = 0;
    n->L.clear();
    for (const D& e : d) {
        Layer l{e.type, e.cin, e.cout, e.level, 0, 0};
        l.w = off;
        off += l.taps() * l.cin * l.cout;
        l.b = off;
        off += l.cout;
        off = (off + 7) / 8 * 8;
        n->L.push_back(l);
    }
    n->np = off;
}

Vol level_vol(Vol v0, int level) {
    Vol v = v0;
    for (int i = 0; i < level; ++i) v = half_vol(v);
    return v;
}

// Activation storage for volume v0.
void ensure_buffers(PNet* n, Vol v0, bool train) {
    for (int i = 0; i < 12; ++i) {
        const Layer& l = n->L[i];
        const size_t pts = (size_t)level_vol(v0, l.level).n();
        if (l.type == L_HEAD) {
            n->y.get(pts);
            continue;
        }
        n->z[i].get(pts * l.cout);
        n->a[i].get(pts * l.cout);
        if (train) n->dz[i].get(pts * l.cout);
    }
    n->x.get((size_t)v0.n() * n->in_ch);
    n->wT.get(27 * 32 * 32);
    n->red.get(8);
}

void forward(dft_context* ctx, PNet* n, Vol v0, const bf16* x) {
    const Vol v1 = half_vol(v0), v2 = half_vol(v1);
    const bf16* P = n->pb.p;
    const float* F = n->p.p;
    auto W = [&](int i) { return P + n->L[i].w; };
    auto B = [&](int i) { return F + n->L[i].b; };
    const int ew = 256;
    const bool tc = ctx->net_tensor_cores != 0;
    int* err = n->tc_err.get(1);
    auto c16 = [&](const bf16* in, int i) {
        if (tc) launch_conv3_tc<16, 16>(ctx, v0, in, W(i), B(i), n->z[i].p, n->a[i].p, err);
        else launch_conv3<16, 16, bf16, false>(ctx, v0, in, W(i), B(i), n->z[i].p, n->a[i].p, nullptr, nullptr, nullptr);
    };
    auto c32 = [&](Vol vv, const bf16* in, int i) {
        if (tc) launch_conv3_tc<32, 32>(ctx, vv, in, W(i), B(i), n->z[i].p, n->a[i].p, err);
        else launch_conv3<32, 32, bf16, false>(ctx, vv, in, W(i), B(i), n->z[i].p, n->a[i].p, nullptr, nullptr, nullptr);
    };
    if (n->in_ch == 2)
        launch_conv3<2, 16, bf16, false>(ctx, v0, x, W(0), B(0), n->z[0].p, n->a[0].p, nullptr, nullptr, nullptr);
    else
        fail(DFT_INVALID_ARGUMENT, "the network takes 2 input channels");
    c16(n->a[0].p, 1);
    down_fwd_kernel<16, 32><<<blocks_for(ctx, v1.n()), ew, 0, ctx->stream>>>(v0, v1, n->a[1].p, W(2), B(2), n->z[2].p,
                                                                             n->a[2].p);
    c32(v1, n->a[2].p, 3);
    down_fwd_kernel<32, 32><<<blocks_for(ctx, v2.n()), ew, 0, ctx->stream>>>(v1, v2, n->a[3].p, W(4), B(4), n->z[4].p,
                                                                             n->a[4].p);
    c32(v2, n->a[4].p, 5);
    c32(v2, n->a[5].p, 6);
    up_fwd_kernel<32, 32><<<blocks_for(ctx, v1.n()), ew, 0, ctx->stream>>>(v1, v2, n->a[6].p, W(7), B(7), n->a[3].p,
                                                                           n->z[7].p, n->a[7].p);
    c32(v1, n->a[7].p, 8);
    up_fwd_kernel<32, 16><<<blocks_for(ctx, v0.n()), ew, 0, ctx->stream>>>(v0, v1, n->a[8].p, W(9), B(9), n->a[1].p,
                                                                           n->z[9].p, n->a[9].p);
    c16(n->a[9].p, 10);
    head_fwd_kernel<16><<<blocks_for(ctx, v0.n()), ew, 0, ctx->stream>>>(v0.n(), n->a[10].p, W(11), B(11), n->y.p);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 5);
}

// Loss on the error e = y - t over interior points: w_mse * mean(e^2) + mean((J^k e)^2), J one
// Jacobi sweep on the error (k = 0: plain MSE).  The second term weighs the smooth part of
// the error, which is what a Jacobi solve from the start has to remove sweep by sweep.
struct LossSpec {
    int k = 0;
    float w_mse = 1.f;
    float cx = 0.f, cy = 0.f, cz = 0.f, iden = 0.f;
};

LossSpec loss_spec(const Grid& g, int k, double w_mse) {
    LossSpec L;
    L.k = k;
    L.w_mse = (float)w_mse;
    L.cx = (float)g.ix2;
    L.cy = (float)g.iy2;
    L.cz = (float)g.iz2;
    L.iden = (float)(1.0 / (2.0 * (g.ix2 + g.iy2 + g.iz2)));
    return L;
}

// Adds the loss to *red; writes dL/dy into dy when dy is not null.  y null = zero correction.
void loss_dy(dft_context* ctx, PNet* n, Vol v0, const LossSpec& L, const float* y, const float* t, float* dy,
             double* red) {
    const long long N = v0.n();
    const long long nint = (long long)std::max(v0.nx - 2, 1) * std::max(v0.ny - 2, 1) * std::max(v0.nz - 2, 1);
    const double inv = 1.0 / (double)nint;
    float* e0 = n->e0.get((size_t)N);
    const int nb = blocks_for(ctx, N);
    err_init_kernel<<<nb, 256, 0, ctx->stream>>>(v0, y, t, e0);
    sq_sum_kernel<<<nb, 256, 0, ctx->stream>>>(N, e0, L.w_mse * inv, red, nullptr, 0.f);
    count_launch(ctx, 2);
    const float* add = nullptr;
    if (L.k > 0) {
        float* b[2] = {n->e1.get((size_t)N), n->e2.get((size_t)N)};
        const float* src = e0;
        int cur = 0;
        for (int i = 0; i < L.k; ++i) {
            err_jacobi_kernel<<<nb, 256, 0, ctx->stream>>>(v0, L.cx, L.cy, L.cz, L.iden, src, b[cur]);
            src = b[cur];
            cur ^= 1;
        }
        // src = J^k e in b[cur ^ 1]; gradient seed 2/n * J^k e in b[cur]
        sq_sum_kernel<<<nb, 256, 0, ctx->stream>>>(N, src, inv, red, dy ? b[cur] : nullptr, (float)(2.0 * inv));
        count_launch(ctx, L.k + 1);
        if (dy) {
            for (int i = 0; i < L.k; ++i) {
                err_jacobi_kernel<<<nb, 256, 0, ctx->stream>>>(v0, L.cx, L.cy, L.cz, L.iden, b[cur], b[cur ^ 1]);
                cur ^= 1;
            }
            count_launch(ctx, L.k);
            add = b[cur];
        }
    }
    if (dy) {
        axpy_kernel<<<nb, 256, 0, ctx->stream>>>(N, (float)(2.0 * L.w_mse * inv), e0, add, dy);
        count_launch(ctx);
    }
    DFT_LAUNCH_CHECK();
}

// Adds the gradient of the loss against target t (device, N0) to n->g; adds the loss to n->red[0].
void backward(dft_context* ctx, PNet* n, Vol v0, const bf16* x, const float* t, const LossSpec& L) {
    const Vol v1 = half_vol(v0), v2 = half_vol(v1);
    const bf16* P = n->pb.p;
    float* G = n->g.p;
    auto W = [&](int i) { return P + n->L[i].w; };
    auto GW = [&](int i) { return G + n->L[i].w; };
    auto GB = [&](int i) { return G + n->L[i].b; };
    const int ew = 256;
    const bool tc = ctx->net_tensor_cores != 0;
    int* err = n->tc_err.get(1);
    // data gradient of a square 3x3x3 layer (weights already flipped into n->wT)
    auto conv_bwd16 = [&](Vol vv, const float* dzin, float* gout, const bf16* zprev) {
        if (tc) launch_conv3_tc_bwd<16>(ctx, n, vv, dzin, n->wT.p, gout, zprev, err);
        else launch_conv3<16, 16, float, true>(ctx, vv, dzin, n->wT.p, nullptr, nullptr, nullptr, gout, nullptr, zprev);
    };
    auto conv_bwd32 = [&](Vol vv, const float* dzin, float* gout, const bf16* zprev) {
        if (tc) launch_conv3_tc_bwd<32>(ctx, n, vv, dzin, n->wT.p, gout, zprev, err);
        else launch_conv3<32, 32, float, true>(ctx, vv, dzin, n->wT.p, nullptr, nullptr, nullptr, gout, nullptr, zprev);
    };
    const long long nint = (long long)std::max(v0.nx - 2, 1) * std::max(v0.ny - 2, 1) * std::max(v0.nz - 2, 1);
    float* dy = n->dy.get((size_t)v0.n());
    loss_dy(ctx, n, v0, L, n->y.p, t, dy, n->red.p);
    head_bwd_kernel<16><<<blocks_for(ctx, v0.n()), ew, 0, ctx->stream>>>(v0.n(), dy, n->a[10].p, n->z[10].p, W(11),
                                                                         n->dz[10].p, GW(11), GB(11));
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    // c11: conv3 16->16 at level 0
    launch_wgrad<16, 16>(ctx, v0, n->a[9].p, n->dz[10].p, GW(10), GB(10));
    flip(ctx, 16, 16, W(10), n->wT.p);
    conv_bwd16(v0, n->dz[10].p, n->dz[9].p, n->z[9].p);
    // c10: up 32->16 (+ skip a1)
    pair_wgrad_kernel<32, 16, true><<<blocks_for(ctx, v1.n(), 16), 256, 0, ctx->stream>>>(v0, v1, n->a[8].p,
                                                                                          n->dz[9].p, GW(9), GB(9));
    up_bwd_kernel<32, 16><<<blocks_for(ctx, v1.n()), ew, 0, ctx->stream>>>(v0, v1, n->dz[9].p, W(9), n->z[8].p,
                                                                           n->dz[8].p);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    // c9: conv3 32->32 at level 1
    launch_wgrad<32, 32>(ctx, v1, n->a[7].p, n->dz[8].p, GW(8), GB(8));
    flip(ctx, 32, 32, W(8), n->wT.p);
    conv_bwd32(v1, n->dz[8].p, n->dz[7].p, n->z[7].p);
    // c8: up 32->32 (+ skip a3)
    pair_wgrad_kernel<32, 32, true><<<blocks_for(ctx, v2.n(), 16), 256, 0, ctx->stream>>>(v1, v2, n->a[6].p,
                                                                                          n->dz[7].p, GW(7), GB(7));
    up_bwd_kernel<32, 32><<<blocks_for(ctx, v2.n()), ew, 0, ctx->stream>>>(v1, v2, n->dz[7].p, W(7), n->z[6].p,
                                                                           n->dz[6].p);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    // c7, c6: conv3 32->32 at level 2
    launch_wgrad<32, 32>(ctx, v2, n->a[5].p, n->dz[6].p, GW(6), GB(6));
    flip(ctx, 32, 32, W(6), n->wT.p);
    conv_bwd32(v2, n->dz[6].p, n->dz[5].p, n->z[5].p);
    launch_wgrad<32, 32>(ctx, v2, n->a[4].p, n->dz[5].p, GW(5), GB(5));
    flip(ctx, 32, 32, W(5), n->wT.p);
    conv_bwd32(v2, n->dz[5].p, n->dz[4].p, n->z[4].p);
    // c5: down 32->32; a3 also feeds the skip of c8
    pair_wgrad_kernel<32, 32, false><<<blocks_for(ctx, v2.n(), 16), 256, 0, ctx->stream>>>(v1, v2, n->a[3].p,
                                                                                           n->dz[4].p, GW(4), GB(4));
    down_bwd_kernel<32, 32><<<blocks_for(ctx, v1.n()), ew, 0, ctx->stream>>>(v1, v2, n->dz[4].p, W(4), n->dz[7].p,
                                                                             n->z[3].p, n->dz[3].p);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    // c4: conv3 32->32 at level 1
    launch_wgrad<32, 32>(ctx, v1, n->a[2].p, n->dz[3].p, GW(3), GB(3));
    flip(ctx, 32, 32, W(3), n->wT.p);
    conv_bwd32(v1, n->dz[3].p, n->dz[2].p, n->z[2].p);
    // c3: down 16->32; a1 also feeds the skip of c10
    pair_wgrad_kernel<16, 32, false><<<blocks_for(ctx, v1.n(), 16), 256, 0, ctx->stream>>>(v0, v1, n->a[1].p,
                                                                                           n->dz[2].p, GW(2), GB(2));
    down_bwd_kernel<16, 32><<<blocks_for(ctx, v0.n()), ew, 0, ctx->stream>>>(v0, v1, n->dz[2].p, W(2), n->dz[9].p,
                                                                             n->z[1].p, n->dz[1].p);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    // c2: conv3 16->16 at level 0
    launch_wgrad<16, 16>(ctx, v0, n->a[0].p, n->dz[1].p, GW(1), GB(1));
    flip(ctx, 16, 16, W(1), n->wT.p);
    conv_bwd16(v0, n->dz[1].p, n->dz[0].p, n->z[0].p);
    // c1: weights only
    launch_wgrad<2, 16>(ctx, v0, x, n->dz[0].p, GW(0), GB(0));
}

// Reads the tensor-core convolutions' error flag (synchronises the stream).
void check_tc(dft_context* ctx, PNet* n) {
    int* h = (int*)pinned(ctx, 1);
    DFT_CUDA(cudaMemcpyAsync(h, n->tc_err.get(1), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    if (*h) fail(DFT_CUDA_ERROR, "tensor-core convolution: mbarrier wait timed out");
}

void adam_step(dft_context* ctx, PNet* n, float lr, float gscale) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    n->step += 1;
    const float c1 = 1.f / (1.f - std::pow(b1, (float)n->step));
    const float c2 = 1.f / (1.f - std::pow(b2, (float)n->step));
    adam_kernel<<<blocks_for(ctx, (long long)n->np), 256, 0, ctx->stream>>>((long long)n->np, n->p.p, n->g.p, n->m.p,
                                                                            n->v.p, n->pb.p, lr, b1, b2, eps, c1, c2,
                                                                            gscale);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
}

void net_input(dft_context* ctx, PNet* n, const Grid& g, const double* rho, const double* vup, const double* s,
               bf16* x) {
    const double h2 = (g.dx * g.dx + g.dy * g.dy + g.dz * g.dz) / 3.0;
    build_input_kernel<<<blocks_for(ctx, g.N), 256, 0, ctx->stream>>>(g.N, rho, vup, s, h2, x);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    (void)n;
}

}  // namespace


dft_pnet* pnet_create(dft_context* ctx, int in_channels, unsigned long long seed) {
    if (in_channels != 2) fail(DFT_INVALID_ARGUMENT, "the Poisson network takes 2 input channels");
    auto* n = new dft_pnet();
    n->ctx = ctx;
    n->in_ch = in_channels;
    try {
        build_layers(n);
        std::vector<float> h(n->np, 0.f);
        std::mt19937_64 rng(seed);
        for (const Layer& l : n->L) {
            const double fan_in = (double)l.taps() * l.cin;
            // He-uniform for SiLU layers; the head starts near zero so the untrained network
            // leaves the coarse start unchanged
            const double b = l.type == L_HEAD ? 1e-3 : std::sqrt(6.0 / fan_in);
            std::uniform_real_distribution<double> u(-b, b);
            for (size_t e = 0; e < l.taps() * l.cin * l.cout; ++e) h[l.w + e] = (float)u(rng);
        }
        n->p.get(n->np);
        n->g.get(n->np);
        n->m.get(n->np);
        n->v.get(n->np);
        n->pb.get(n->np);
        DFT_CUDA(cudaMemsetAsync(n->tc_err.get(1), 0, sizeof(int), ctx->stream));
        DFT_CUDA(cudaMemsetAsync(n->m.p, 0, n->np * 4, ctx->stream));
        DFT_CUDA(cudaMemsetAsync(n->v.p, 0, n->np * 4, ctx->stream));
        pnet_set_params(ctx, n, h.data());
    } catch (...) {
        delete n;
        throw;
    }
    return n;
}

void pnet_destroy(dft_pnet* net) { delete net; }

size_t pnet_num_params(const dft_pnet* net) { return net->np; }

void pnet_get_params(dft_context* ctx, dft_pnet* n, float* host) {
    DFT_CUDA(cudaMemcpyAsync(host, n->p.p, n->np * 4, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
}

void pnet_set_params(dft_context* ctx, dft_pnet* n, const float* host) {
    DFT_CUDA(cudaMemcpyAsync(n->p.p, host, n->np * 4, cudaMemcpyHostToDevice, ctx->stream));
    to_bf16_kernel<<<blocks_for(ctx, (long long)n->np), 256, 0, ctx->stream>>>((long long)n->np, n->p.p, n->pb.p);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    sync(ctx);
}

void pnet_loss_grad(dft_context* ctx, dft_pnet* n, int nx, int ny, int nz, const float* x_host, const float* t_host,
                    double* loss, float* grad_host, float* y_host) {
    if (nx < 3 || ny < 3 || nz < 3) fail(DFT_INVALID_ARGUMENT, "volume must have at least 3 points per axis");
    const Vol v0{nx, ny, nz};
    ensure_buffers(n, v0, true);
    const size_t N = (size_t)v0.n();
    std::vector<__nv_bfloat16> xb(N * n->in_ch);
    for (size_t e = 0; e < xb.size(); ++e) xb[e] = __float2bfloat16_rn(x_host[e]);
    DFT_CUDA(cudaMemcpyAsync(n->x.p, xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, ctx->stream));
    float* t = n->t.get(N);
    DFT_CUDA(cudaMemcpyAsync(t, t_host, N * 4, cudaMemcpyHostToDevice, ctx->stream));
    DFT_CUDA(cudaMemsetAsync(n->g.p, 0, n->np * 4, ctx->stream));
    DFT_CUDA(cudaMemsetAsync(n->red.p, 0, 8, ctx->stream));
    forward(ctx, n, v0, n->x.p);
    backward(ctx, n, v0, n->x.p, t, LossSpec{});
    if (grad_host) DFT_CUDA(cudaMemcpyAsync(grad_host, n->g.p, n->np * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (y_host) DFT_CUDA(cudaMemcpyAsync(y_host, n->y.p, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
    double* h = pinned(ctx, 1);
    DFT_CUDA(cudaMemcpyAsync(h, n->red.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    if (loss) *loss = h[0];
    check_tc(ctx, n);
}

void pnet_correct(dft_context* ctx, dft_pnet* net, const Grid& g, const double* rho, double* v,
                  const double* scale_dev) {
    const Vol v0{g.nx, g.ny, g.nz};
    ensure_buffers(net, v0, false);
    net_input(ctx, net, g, rho, v, scale_dev, net->x.p);
    forward(ctx, net, v0, net->x.p);
    combine_kernel<<<blocks_for(ctx, g.N), 256, 0, ctx->stream>>>(g, v, net->y.p, scale_dev, v);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    check_tc(ctx, net);
}

void pnet_train_poisson(dft_context* ctx, dft_pnet* n, const dft_pnet_train_opts* o, dft_pnet_train_report* rep) {
    using Clock = std::chrono::steady_clock;
    if (!o || !rep) fail(DFT_INVALID_ARGUMENT, "NULL options or report");
    if (o->samples < 2 || o->validation < 1 || o->validation >= o->samples || o->epochs < 1 || o->batch < 1 ||
        o->smooth_sweeps < 0 || o->smooth_sweeps > 4096 || !(o->mse_weight >= 0) ||
        o->ngrids < 1 || o->ngrids > 4 || !(o->lr > 0) || o->lr_min < 0 || o->target_max_sweeps < 1)
        fail(DFT_INVALID_ARGUMENT, "invalid training options");
    std::vector<Grid> grids;
    Vol vmax{0, 0, 0};
    for (int i = 0; i < o->ngrids; ++i) {
        grids.push_back(make_grid(&o->grids[i]));
        const Vol v{grids.back().nx, grids.back().ny, grids.back().nz};
        if (v.nx < 3 || v.ny < 3 || v.nz < 3) fail(DFT_INVALID_ARGUMENT, "training grids need an interior");
        if (v.n() > vmax.n()) vmax = v;
    }
    ensure_buffers(n, vmax, true);
    // ---- data: synthetic densities, coarse starts and Jacobi targets
    const auto t0 = Clock::now();
    struct Sample {
        int gi = 0;
        DBuf<bf16> x;
        DBuf<float> t;
    };
    std::vector<std::unique_ptr<Sample>> data;
    DBuf<double> rho, vt, vup, slab;
    long target_sweeps = 0;
    for (int s = 0; s < o->samples; ++s) {
        auto smp = std::make_unique<Sample>();
        smp->gi = s % o->ngrids;
        const Grid& g = grids[smp->gi];
        double* r = rho.get((size_t)g.N);
        double* v = vt.get((size_t)g.N);
        double* u = vup.get((size_t)g.N);
        synthetic_density(ctx, g, o->seed * 0x9E3779B97F4A7C15ULL + (unsigned long long)s, o->kmin, o->kmax, o->wmin,
                          o->wmax, o->ne_min, o->ne_max, r);
        double* sdev = nullptr;
        coarse_start(ctx, slab.get(coarse_slab_doubles(g)), g, r, u, &sdev);
        // target: the Jacobi fixed point to target_tol, reached by multigrid cycles from the
        // coarse start and finished by Jacobi sweeps under the stop rule
        DFT_CUDA(cudaMemcpyAsync(v, u, sizeof(double) * (size_t)g.N, cudaMemcpyDeviceToDevice, ctx->stream));
        multigrid(ctx, g, r, v, 0.5 * o->target_tol, 100, nullptr);
        target_sweeps += hartree(ctx, g, r, v, o->target_tol, o->target_max_sweeps, v).sweeps;
        bf16* x = smp->x.get((size_t)g.N * 2);
        float* t = smp->t.get((size_t)g.N);
        net_input(ctx, n, g, r, u, sdev, x);
        build_target_kernel<<<blocks_for(ctx, g.N), 256, 0, ctx->stream>>>(g, v, u, sdev, t);
        DFT_LAUNCH_CHECK();
        count_launch(ctx);
        data.push_back(std::move(smp));
    }
    sync(ctx);
    rep->seconds_data = std::chrono::duration<double>(Clock::now() - t0).count();
    rep->mean_target_sweeps = (double)target_sweeps / o->samples;
    // ---- training
    const int ntrain = o->samples - o->validation;
    const int spe = (ntrain + o->batch - 1) / o->batch;
    const long total = (long)spe * o->epochs;
    std::mt19937_64 rng(o->seed ^ 0x5DEECE66DULL);
    std::vector<int> order(ntrain);
    std::iota(order.begin(), order.end(), 0);
    double* h = pinned(ctx, 2);
    const auto t1 = Clock::now();
    long step = 0;
    for (int ep = 0; ep < o->epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        DFT_CUDA(cudaMemsetAsync(n->red.p, 0, 8, ctx->stream));
        for (int b0 = 0; b0 < ntrain; b0 += o->batch) {
            const int nb = std::min(o->batch, ntrain - b0);
            DFT_CUDA(cudaMemsetAsync(n->g.p, 0, n->np * 4, ctx->stream));
            for (int b = 0; b < nb; ++b) {
                const Sample& smp = *data[order[b0 + b]];
                const Grid& g = grids[smp.gi];
                const Vol v0{g.nx, g.ny, g.nz};
                forward(ctx, n, v0, smp.x.p);
                backward(ctx, n, v0, smp.x.p, smp.t.p, loss_spec(g, o->smooth_sweeps, o->mse_weight));
            }
            const double cosf_ = 0.5 * (1.0 + std::cos(3.14159265358979323846 * (double)step / (double)total));
            adam_step(ctx, n, (float)(o->lr_min + (o->lr - o->lr_min) * cosf_), 1.f / (float)nb);
            ++step;
        }
        DFT_CUDA(cudaMemcpyAsync(h, n->red.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        const double el = h[0] / ntrain;
        check_tc(ctx, n);
        if (ep == 0) rep->train_loss_first_epoch = el;
        rep->train_loss_last_epoch = el;
        if (rep->epoch_loss && ep < rep->epoch_loss_capacity) rep->epoch_loss[ep] = el;
        if (o->verbose) fprintf(stderr, "[pnet] epoch %d loss %.6e\n", ep + 1, el);
    }
    sync(ctx);
    rep->seconds_train = std::chrono::duration<double>(Clock::now() - t1).count();
    rep->steps = (int)step;
    rep->ms_per_step = step ? 1e3 * rep->seconds_train / step : 0.0;
    // ---- validation: network vs the coarse start alone (zero correction)
    double* red2 = n->red.p;  // holds 8 doubles
    DFT_CUDA(cudaMemsetAsync(red2, 0, 16, ctx->stream));
    for (int s = ntrain; s < o->samples; ++s) {
        const Sample& smp = *data[s];
        const Grid& g = grids[smp.gi];
        const Vol v0{g.nx, g.ny, g.nz};
        const LossSpec L = loss_spec(g, o->smooth_sweeps, o->mse_weight);
        forward(ctx, n, v0, smp.x.p);
        loss_dy(ctx, n, v0, L, n->y.p, smp.t.p, nullptr, red2);
        loss_dy(ctx, n, v0, L, nullptr, smp.t.p, nullptr, red2 + 1);
    }
    DFT_CUDA(cudaMemcpyAsync(h, red2, 16, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    rep->val_loss = h[0] / o->validation;
    rep->val_loss_coarse = h[1] / o->validation;
}


// ---- learned Davidson preconditioner ------------------------------------------------------
// The preconditioning equation of the block eigensolver is (T + sigma) t = r (T = -1/2 lap_h,
// zero outside the box).  One batched multigrid cycle gives t0; the network, fed the scaled
// residual and t0, predicts the rest of the way to the equation's solution on the interior:
// t = t0 + s net([2 h^2 r / s, t0 / s]), s = max |t0| (the equation is linear, so the scaled
// problem looks the same for every band).

void pnet_precondition(dft_context* ctx, dft_pnet* n, const Grid& g, const double* R, long long ld, const int* active,
                       int na, double* T) {
    if (na <= 0) return;
    const Vol v0{g.nx, g.ny, g.nz};
    ensure_buffers(n, v0, false);
    unsigned long long* sb = n->sbits.get(1);
    const double c = 2.0 * (g.dx * g.dx + g.dy * g.dy + g.dz * g.dz) / 3.0;
    const int nb = blocks_for(ctx, g.N);
    for (int a = 0; a < na; ++a) {
        const double* r = R + (long long)active[a] * ld;
        double* t = T + (long long)a * ld;
        DFT_CUDA(cudaMemsetAsync(sb, 0, sizeof(unsigned long long), ctx->stream));
        absmax_kernel<<<nb, 256, 0, ctx->stream>>>(g.N, t, sb);
        pc_input_kernel<<<nb, 256, 0, ctx->stream>>>(g.N, r, t, sb, c, n->x.p);
        forward(ctx, n, v0, n->x.p);
        pc_apply_kernel<<<nb, 256, 0, ctx->stream>>>(g, n->y.p, sb, t);
        DFT_LAUNCH_CHECK();
        count_launch(ctx, 3);
    }
    check_tc(ctx, n);
}

namespace {
// residual bands harvested from the plain eigensolver's iterations
struct Harvest {
    dft_context* ctx;
    long long N;
    int want, got = 0;
    double* R;                  // want x N
    std::vector<double> sigma;  // max(-theta, 1)
};
void harvest_residuals(void* user, const double* R, long long ld, const int* active, int na, const double* theta) {
    auto* h = (Harvest*)user;
    for (int a = 0; a < na && h->got < h->want; ++a, ++h->got) {
        DFT_CUDA(cudaMemcpyAsync(h->R + (long long)h->got * h->N, R + (long long)active[a] * ld,
                                 sizeof(double) * (size_t)h->N, cudaMemcpyDeviceToDevice, h->ctx->stream));
        h->sigma.push_back(std::max(-theta[active[a]], 1.0));
    }
}
}  // namespace

void pnet_train_precond(dft_context* ctx, dft_pnet* n, const Grid& g, const double* V, int nocc, int nbands,
                        const dft_pnet_train_opts* o, dft_pnet_train_report* rep) {
    using Clock = std::chrono::steady_clock;
    if (!o || !rep) fail(DFT_INVALID_ARGUMENT, "NULL options or report");
    if (o->samples < 3 || o->validation < 1 || o->validation >= o->samples || o->epochs < 1 || o->batch < 1 ||
        !(o->lr > 0) || o->lr_min < 0 || o->target_max_sweeps < 2)
        fail(DFT_INVALID_ARGUMENT, "invalid training options");
    if (g.nx < 8 || g.ny < 8 || g.nz < 8) fail(DFT_INVALID_ARGUMENT, "training grid too small");
    const auto t0 = Clock::now();
    const long long N = g.N;
    // ---- data: the plain solver's residual bands in V (multigrid preconditioner), then per band
    // one cycle (the network's input) and target_max_sweeps cycles of refinement (its target)
    DBuf<double> Rs, X0, Xs, res, e, sig, psi;
    Harvest hv{ctx, N, o->samples};
    hv.R = Rs.get((size_t)o->samples * N);
    EigOpts eo;
    eo.tol = o->target_tol > 0 ? o->target_tol : 1e-7;
    eo.max_iterations = 400;
    eo.precond_steps = -1;
    eo.harvest = harvest_residuals;
    eo.harvest_user = &hv;
    std::vector<double> eig(nbands), rn(nbands);
    double* pp = psi.get((size_t)nbands * N);
    try {
        solve_orbitals(ctx, g, V, nocc, nbands, pp, N, false, eig.data(), rn.data(), eo);
    } catch (const Error& err) {
        if (err.status != DFT_NOT_CONVERGED) throw;  // enough residuals may have been harvested anyway
    }
    const int ns = hv.got;
    if (ns < o->validation + 2) fail(DFT_INVALID_ARGUMENT, "the eigensolver produced only %d residual bands", ns);
    double* sd = sig.get((size_t)ns);
    DFT_CUDA(cudaMemcpyAsync(sd, hv.sigma.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, ctx->stream));
    double* x0 = X0.get((size_t)ns * N);
    double* xs = Xs.get((size_t)ns * N);
    double* rr = res.get((size_t)ns * N);
    double* ee = e.get((size_t)ns * N);
    helmholtz_refine(ctx, g, hv.R, ns, sd, x0, N, 1, rr, ee);
    helmholtz_refine(ctx, g, hv.R, ns, sd, xs, N, (int)o->target_max_sweeps, rr, ee);
    const Vol v0{g.nx, g.ny, g.nz};
    ensure_buffers(n, v0, true);
    struct Sample {
        DBuf<bf16> x;
        DBuf<float> t;
    };
    std::vector<std::unique_ptr<Sample>> data;
    unsigned long long* sb = n->sbits.get(1);
    const double c = 2.0 * (g.dx * g.dx + g.dy * g.dy + g.dz * g.dz) / 3.0;
    const int nbk = blocks_for(ctx, N);
    for (int q = 0; q < ns; ++q) {
        auto smp = std::make_unique<Sample>();
        DFT_CUDA(cudaMemsetAsync(sb, 0, sizeof(unsigned long long), ctx->stream));
        absmax_kernel<<<nbk, 256, 0, ctx->stream>>>(N, x0 + (long long)q * N, sb);
        pc_input_kernel<<<nbk, 256, 0, ctx->stream>>>(N, hv.R + (long long)q * N, x0 + (long long)q * N, sb, c,
                                                       smp->x.get((size_t)N * 2));
        pc_target_kernel<<<nbk, 256, 0, ctx->stream>>>(g, xs + (long long)q * N, x0 + (long long)q * N, sb,
                                                        smp->t.get((size_t)N));
        DFT_LAUNCH_CHECK();
        count_launch(ctx, 3);
        data.push_back(std::move(smp));
    }
    sync(ctx);
    rep->seconds_data = std::chrono::duration<double>(Clock::now() - t0).count();
    rep->mean_target_sweeps = (double)o->target_max_sweeps;
    // ---- training: mean squared error of the correction over interior points
    const int nval = std::min(o->validation, ns - 2);
    const int ntrain = ns - nval;
    const int spe = (ntrain + o->batch - 1) / o->batch;
    const long total = (long)spe * o->epochs;
    std::mt19937_64 rng(o->seed ^ 0x2545F4914F6CDD1DULL);
    std::vector<int> order(ntrain);
    std::iota(order.begin(), order.end(), 0);
    double* h = pinned(ctx, 2);
    const LossSpec L = loss_spec(g, 0, 1.0);
    const auto t1 = Clock::now();
    long step = 0;
    for (int ep = 0; ep < o->epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        DFT_CUDA(cudaMemsetAsync(n->red.p, 0, 8, ctx->stream));
        for (int b0 = 0; b0 < ntrain; b0 += o->batch) {
            const int nb = std::min(o->batch, ntrain - b0);
            DFT_CUDA(cudaMemsetAsync(n->g.p, 0, n->np * 4, ctx->stream));
            for (int b = 0; b < nb; ++b) {
                const Sample& smp = *data[order[b0 + b]];
                forward(ctx, n, v0, smp.x.p);
                backward(ctx, n, v0, smp.x.p, smp.t.p, L);
            }
            const double cosf_ = 0.5 * (1.0 + std::cos(3.14159265358979323846 * (double)step / (double)total));
            adam_step(ctx, n, (float)(o->lr_min + (o->lr - o->lr_min) * cosf_), 1.f / (float)nb);
            ++step;
        }
        DFT_CUDA(cudaMemcpyAsync(h, n->red.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
        sync(ctx);
        const double el = h[0] / ntrain;
        check_tc(ctx, n);
        if (ep == 0) rep->train_loss_first_epoch = el;
        rep->train_loss_last_epoch = el;
        if (rep->epoch_loss && ep < rep->epoch_loss_capacity) rep->epoch_loss[ep] = el;
        if (o->verbose) fprintf(stderr, "[pnet precond] epoch %d loss %.6e\n", ep + 1, el);
    }
    sync(ctx);
    rep->seconds_train = std::chrono::duration<double>(Clock::now() - t1).count();
    rep->steps = (int)step;
    rep->ms_per_step = step ? 1e3 * rep->seconds_train / step : 0.0;
    // ---- validation: network vs one multigrid cycle alone (zero correction)
    double* red2 = n->red.p;
    DFT_CUDA(cudaMemsetAsync(red2, 0, 16, ctx->stream));
    for (int q = ntrain; q < ns; ++q) {
        const Sample& smp = *data[q];
        forward(ctx, n, v0, smp.x.p);
        loss_dy(ctx, n, v0, L, n->y.p, smp.t.p, nullptr, red2);
        loss_dy(ctx, n, v0, L, nullptr, smp.t.p, nullptr, red2 + 1);
    }
    DFT_CUDA(cudaMemcpyAsync(h, red2, 16, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    rep->val_loss = h[0] / nval;
    rep->val_loss_coarse = h[1] / nval;
}

}  // namespace dftb
