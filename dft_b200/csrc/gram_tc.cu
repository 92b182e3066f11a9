// Mixed-precision Gram products on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// C (ka x kb) = dV * A^T B for tall-skinny band blocks (A_i, B_j contiguous over N grid points).
// Each FP64 input x is split into two TF32 numbers, x ~ hi + lo (hi = TF32-rounded x,
// lo = TF32(x - hi)), and the product is formed as hi*hi + hi*lo + lo*hi with FP32
// accumulation in tensor memory (TMEM): relative error ~1e-6, the "FP32-level" precision the
// block eigensolver uses while residuals are large.  Per block:
//   * 256 threads stage a 32-point K slice of A (128 rows) and B (<= 256 rows) from HBM,
//     split them and store hi/lo planes in shared memory in the canonical K-major layout
//     (8-row x 16-byte core matrices, no swizzle), double-buffered; the next slice's FP64
//     values are loaded into registers while the tensor cores consume the current one;
//   * one thread issues 12 tcgen05.mma.kind::tf32 (4 K=8 steps x 3 products) into a
//     128 x N FP32 accumulator in TMEM and commits them to an mbarrier;
//   * after its K range the block reads the accumulator back with tcgen05.ld (each warp its
//     32 TMEM lanes) and writes FP64 partial sums; a deterministic FP64 reduction over blocks
//     (gram_reduce_kernel in davidson.cu) finishes the product.
// Every mbarrier wait is bounded; a block that gives up sets an error flag, waits (bounded)
// for its own MMAs, frees its TMEM and returns.
#include <cstdint>
#include <vector>

#include "ops.h"

namespace dftb {

namespace {

constexpr int TC_THREADS = 256;
constexpr int TC_M = 128;     // accumulator rows (A vectors per tile)
constexpr int TC_KT = 32;     // points per K slice
constexpr int TC_NMAX = 256;  // accumulator columns (B vectors per tile)
constexpr long long TC_SPIN_LIMIT = 1LL << 22;  // try_wait polls before a block gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// canonical K-major, no-swizzle placement of element (row, k) of an R-row x 32-point slice:
// core matrix (8 rows x 4 fp32) index = (k/4) * (R/8) + row/8, 128 bytes each
__device__ __forceinline__ int kmajor_offset_words(int row, int k, int R) {
    return (((k >> 2) * (R >> 3) + (row >> 3)) << 5) + ((row & 7) << 2) + (k & 3);
}

// UMMA shared-memory matrix descriptor (sm_100: version 1, no swizzle)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version
    return d;                // layout type 0 = SWIZZLE_NONE, base offset 0
}

// instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// bounded wait for the phase with the given parity to complete; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long i = 0; i < TC_SPIN_LIMIT; ++i) {
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

__device__ __forceinline__ void mma_tf32(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    const uint32_t z = 0;  // no output lanes disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        ::"r"(tmem_c), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Gram tile.  grid = (ceil(ka/128), ceil(kb/nt), nchunks); dynamic smem = 2 stages x
// (A hi, A lo: 128 x 32 fp32; B hi, B lo: NC x 32 fp32).  Row r of a slice is read by warp
// r % 8 (one point per lane); each thread holds the next slice's raw FP64 values in
// registers, loaded while the tensor cores work on the current slice.
template <int NC>
__global__ void __launch_bounds__(TC_THREADS, 1)
    gram_tc_kernel(const double* __restrict__ A, long long lda, int ka, const double* __restrict__ B, long long ldb,
                   int kb, int nt, long long n, long long chunk, double* __restrict__ partial,
                   int* __restrict__ error) {
    extern __shared__ __align__(1024) uint32_t sm[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t bar[2];
    constexpr int NW = TC_THREADS / 32;
    constexpr int RA = TC_M / NW, RB = NC / NW;  // rows per warp
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_M, n0 = blockIdx.y * nt;
    const int mrows = min(TC_M, ka - m0), nrows = min(nt, kb - n0);
    const long long p0 = (long long)blockIdx.z * chunk, p1 = min(n, p0 + chunk);
    constexpr int a_words = TC_M * TC_KT, b_words = NC * TC_KT;
    constexpr int stage_words = 2 * a_words + 2 * b_words;
    // TMEM: NC fp32 columns x 128 lanes, allocated by warp 0
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(NC));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_tf32(NC);
    // Thread (warp, lane) owns element (row 8 rg + lane / 4, point 4 kg + lane % 4) of core
    // matrix cm = warp + 8 i (rg = cm / 8, kg = cm % 8): a warp writes one whole 128-byte core
    // matrix per store, so the shared-memory stores are free of bank conflicts.
    double xa[RA], xb[RB];
    const int lr = lane >> 2, lk = lane & 3;
    auto load = [&](long long ps) {
#pragma unroll
        for (int i = 0; i < RA; ++i) {
            const int cm = warp + i * NW, r = (cm >> 3) * 8 + lr;
            const long long pt = ps + (cm & 7) * 4 + lk;
            xa[i] = (r < mrows && pt < p1) ? __ldg(A + (long long)(m0 + r) * lda + pt) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < RB; ++i) {
            const int cm = warp + i * NW, r = (cm >> 3) * 8 + lr;
            const long long pt = ps + (cm & 7) * 4 + lk;
            xb[i] = (r < nrows && pt < p1) ? __ldg(B + (long long)(n0 + r) * ldb + pt) : 0.0;
        }
    };
    if (p0 < p1) load(p0);
    bool ok = true;
    uint32_t phase[2] = {0, 0};
    bool pending[2] = {false, false};
    int step = 0;
    for (long long ps = p0; ps < p1; ps += TC_KT, ++step) {
        const int st = step & 1;
        // the MMAs that last read this stage must be done before it is overwritten
        if (pending[st]) {
            if (!mbar_wait(&bar[st], phase[st])) ok = false;
            phase[st] ^= 1;
            pending[st] = false;
        }
        if (!__syncthreads_and(ok)) break;
        uint32_t* ahi = sm + st * stage_words;
        uint32_t* alo = ahi + a_words;
        uint32_t* bhi = alo + a_words;
        uint32_t* blo = bhi + b_words;
#pragma unroll
        for (int i = 0; i < RA; ++i) {
            const int cm = warp + i * NW;
            const uint32_t h = to_tf32((float)xa[i]);
            const uint32_t l = to_tf32((float)(xa[i] - (double)__uint_as_float(h)));
            const int o = (((cm & 7) * (TC_M / 8) + (cm >> 3)) << 5) + lane;  // = kmajor_offset_words(row, k, TC_M)
            ahi[o] = h;
            alo[o] = l;
        }
#pragma unroll
        for (int i = 0; i < RB; ++i) {
            const int cm = warp + i * NW;
            const uint32_t h = to_tf32((float)xb[i]);
            const uint32_t l = to_tf32((float)(xb[i] - (double)__uint_as_float(h)));
            const int o = (((cm & 7) * (NC / 8) + (cm >> 3)) << 5) + lane;
            bhi[o] = h;
            blo[o] = l;
        }
        // generic-proxy smem writes -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t lbo_a = (TC_M / 8) * 128, lbo_b = (uint32_t)(NC / 8) * 128, sbo = 128;
            const uint32_t sa_hi = smem_u32(ahi), sa_lo = smem_u32(alo), sb_hi = smem_u32(bhi), sb_lo = smem_u32(blo);
#pragma unroll
            for (int kk = 0; kk < TC_KT / 8; ++kk) {
                // K = 8 tf32 = two 4-element core-matrix columns
                const uint32_t oa = kk * 2 * lbo_a, ob = kk * 2 * lbo_b;
                const uint64_t dah = smem_desc(sa_hi + oa, lbo_a, sbo), dal = smem_desc(sa_lo + oa, lbo_a, sbo);
                const uint64_t dbh = smem_desc(sb_hi + ob, lbo_b, sbo), dbl = smem_desc(sb_lo + ob, lbo_b, sbo);
                const uint32_t first = (step == 0 && kk == 0) ? 0u : 1u;
                mma_tf32(tmem, dah, dbh, idesc, first);
                mma_tf32(tmem, dah, dbl, idesc, 1u);
                mma_tf32(tmem, dal, dbh, idesc, 1u);
            }
            mma_commit(&bar[st]);
        }
        pending[st] = true;
        // the next slice's loads overlap the MMAs just issued
        if (ps + TC_KT < p1) load(ps + TC_KT);
    }
    // drain: wait (bounded) for every stage that still has MMAs in flight
    for (int st = 0; st < 2; ++st)
        if (pending[st]) {
            if (!mbar_wait(&bar[st], phase[st])) ok = false;
            phase[st] ^= 1;
        }
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0) atomicExch(error, 1);
    } else if (step > 0) {
        // accumulator row r = A vector m0 + r lives in TMEM lane r: warp w reads lanes
        // 32 (w % 4) .. +31; warps w and w + 4 split the columns
        double* out = partial + (long long)blockIdx.z * ka * kb;
        const int q4 = warp & 3, half = warp >> 2;
        const int row = q4 * 32 + lane;
        constexpr int CH = NC / (NW / 4);
        for (int c0 = half * CH; c0 < half * CH + CH; c0 += 8) {
            uint32_t v[8];
            const uint32_t addr = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < mrows)
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (c0 + q < nrows) out[(long long)(m0 + row) * kb + (n0 + c0 + q)] = (double)__uint_as_float(v[q]);
        }
    } else {
        // empty K range: this block contributes zeros
        double* out = partial + (long long)blockIdx.z * ka * kb;
        for (int e = tid; e < mrows * nrows; e += TC_THREADS)
            out[(long long)(m0 + e / nrows) * kb + (n0 + e % nrows)] = 0.0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NC));
}

// Ring variant of the Gram tile (tuning key "tensor_core_ring"): the FP64 slices are staged
// into a 2-deep shared-memory ring with cp.async (16-byte chunks, zero-filled past the ends),
// so two slices are in flight per block without holding them in registers; each slice is
// then split from shared memory into the TF32 hi/lo planes of one operand buffer (the same
// core-matrix layout and MMAs as gram_tc_kernel).  Needs even leading dimensions and
// 16-byte-aligned A and B; NC <= 128.
constexpr int TR_STAGES = 2;
constexpr int TR_RS = 36;  // doubles per staged row: 32 points + 4 of padding (fewer bank conflicts)

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

template <int NC>
__global__ void __launch_bounds__(TC_THREADS, 1)
    gram_tc_ring_kernel(const double* __restrict__ A, long long lda, int ka, const double* __restrict__ B,
                        long long ldb, int kb, int nt, long long n, long long chunk, double* __restrict__ partial,
                        int* __restrict__ error) {
    extern __shared__ __align__(1024) uint32_t sm[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t bar;
    constexpr int NW = TC_THREADS / 32;
    constexpr int RA = TC_M / NW, RB = NC / NW;
    constexpr int ROWS = TC_M + NC;
    constexpr int a_words = TC_M * TC_KT, b_words = NC * TC_KT;
    uint32_t* ahi = sm;  // one operand buffer: A hi, A lo, B hi, B lo
    uint32_t* alo = ahi + a_words;
    uint32_t* bhi = alo + a_words;
    uint32_t* blo = bhi + b_words;
    double* raw = reinterpret_cast<double*>(blo + b_words);  // TR_STAGES x ROWS x TR_RS
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_M, n0 = blockIdx.y * nt;
    const int mrows = min(TC_M, ka - m0), nrows = min(nt, kb - n0);
    const long long p0 = (long long)blockIdx.z * chunk, p1 = min(n, p0 + chunk);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(NC));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_tf32(NC);
    // stage the slice starting at point ps into ring slot st: ROWS x 16 chunks of 2 doubles
    auto stage = [&](long long ps, int st) {
        double* dst0 = raw + (size_t)st * ROWS * TR_RS;
        for (int c = tid; c < ROWS * 16; c += TC_THREADS) {
            const int row = c >> 4, q = c & 15;
            const long long pt = ps + 2 * q;
            const double* base;
            bool valid;
            if (row < TC_M) {
                valid = row < mrows;
                base = A + (long long)(m0 + (valid ? row : 0)) * lda;
            } else {
                valid = row - TC_M < nrows;
                base = B + (long long)(n0 + (valid ? row - TC_M : 0)) * ldb;
            }
            const long long left = p1 - pt;  // doubles left in this block's range
            const uint32_t bytes = (!valid || left <= 0) ? 0u : (left >= 2 ? 16u : 8u);
            cp_async16(smem_u32(dst0 + (size_t)row * TR_RS + 2 * q), bytes ? base + pt : base, bytes);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    const int nsteps = (int)((p1 - p0 + TC_KT - 1) / TC_KT);
    for (int s0 = 0; s0 < TR_STAGES; ++s0) {
        if (s0 < nsteps) stage(p0 + (long long)s0 * TC_KT, s0);
        else asm volatile("cp.async.commit_group;" ::: "memory");  // keep the group count uniform
    }
    bool ok = true;
    uint32_t phase = 0;
    bool pending = false;
    const int lr = lane >> 2, lk = lane & 3;
    for (int step = 0; step < nsteps; ++step) {
        const int st = step % TR_STAGES;
        // slice `step` has landed (at most TR_STAGES - 1 younger groups still in flight)
        asm volatile("cp.async.wait_group %0;" ::"n"(TR_STAGES - 1) : "memory");
        // the MMAs of the previous slice must be done before the operand buffer is rewritten;
        // after a timed-out wait they count as still in flight (waited for again below)
        if (pending) {
            if (mbar_wait(&bar, phase)) {
                phase ^= 1;
                pending = false;
            } else {
                ok = false;
            }
        }
        if (!__syncthreads_and(ok)) break;
        const double* src = raw + (size_t)st * ROWS * TR_RS;
#pragma unroll
        for (int i = 0; i < RA; ++i) {
            const int cm = warp + i * NW, r = (cm >> 3) * 8 + lr, pt = (cm & 7) * 4 + lk;
            const double x = src[(size_t)r * TR_RS + pt];
            const uint32_t h = to_tf32((float)x);
            const uint32_t l = to_tf32((float)(x - (double)__uint_as_float(h)));
            const int o = (((cm & 7) * (TC_M / 8) + (cm >> 3)) << 5) + lane;
            ahi[o] = h;
            alo[o] = l;
        }
#pragma unroll
        for (int i = 0; i < RB; ++i) {
            const int cm = warp + i * NW, r = (cm >> 3) * 8 + lr, pt = (cm & 7) * 4 + lk;
            const double x = src[(size_t)(TC_M + r) * TR_RS + pt];
            const uint32_t h = to_tf32((float)x);
            const uint32_t l = to_tf32((float)(x - (double)__uint_as_float(h)));
            const int o = (((cm & 7) * (NC / 8) + (cm >> 3)) << 5) + lane;
            bhi[o] = h;
            blo[o] = l;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t lbo_a = (TC_M / 8) * 128, lbo_b = (uint32_t)(NC / 8) * 128, sbo = 128;
            const uint32_t sa_hi = smem_u32(ahi), sa_lo = smem_u32(alo), sb_hi = smem_u32(bhi), sb_lo = smem_u32(blo);
#pragma unroll
            for (int kk = 0; kk < TC_KT / 8; ++kk) {
                const uint32_t oa = kk * 2 * lbo_a, ob = kk * 2 * lbo_b;
                const uint64_t dah = smem_desc(sa_hi + oa, lbo_a, sbo), dal = smem_desc(sa_lo + oa, lbo_a, sbo);
                const uint64_t dbh = smem_desc(sb_hi + ob, lbo_b, sbo), dbl = smem_desc(sb_lo + ob, lbo_b, sbo);
                const uint32_t first = (step == 0 && kk == 0) ? 0u : 1u;
                mma_tf32(tmem, dah, dbh, idesc, first);
                mma_tf32(tmem, dah, dbl, idesc, 1u);
                mma_tf32(tmem, dal, dbh, idesc, 1u);
            }
            mma_commit(&bar);
        }
        pending = true;
        // the ring slot just converted is free: stage the slice TR_STAGES ahead into it (every
        // thread has passed the barrier above, so no one still reads it)
        if (step + TR_STAGES < nsteps) stage(p0 + (long long)(step + TR_STAGES) * TC_KT, st);
        else asm volatile("cp.async.commit_group;" ::: "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    // drain (bounded): the last MMAs, or a second wait for the ones that timed out above
    if (pending && !mbar_wait(&bar, phase)) ok = false;
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0) atomicExch(error, 1);
    } else if (nsteps > 0) {
        double* out = partial + (long long)blockIdx.z * ka * kb;
        const int q4 = warp & 3, half = warp >> 2;
        const int row = q4 * 32 + lane;
        constexpr int CH = NC / (NW / 4);
        for (int c0 = half * CH; c0 < half * CH + CH; c0 += 8) {
            uint32_t v[8];
            const uint32_t addr = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < mrows)
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (c0 + q < nrows) out[(long long)(m0 + row) * kb + (n0 + c0 + q)] = (double)__uint_as_float(v[q]);
        }
    } else {
        double* out = partial + (long long)blockIdx.z * ka * kb;
        for (int e = tid; e < mrows * nrows; e += TC_THREADS)
            out[(long long)(m0 + e / nrows) * kb + (n0 + e % nrows)] = 0.0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NC));
}

template <int NC>
constexpr size_t ring_smem() {
    return sizeof(uint32_t) * (2 * TC_M * TC_KT + 2 * NC * TC_KT) +
           sizeof(double) * (size_t)TR_STAGES * (TC_M + NC) * TR_RS;
}

__global__ void gram_tc_reduce_kernel(int nchunks, int nel, const double* __restrict__ partial, double scale,
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

// Rotation tile: X[n][p] = sum_k V[k][p] Y[k][n] for a 128-point tile (TMEM lanes = points)
// and NC output bands (TMEM columns).  A = the V tile transposed (points x bands), B = Y^T
// (bands-out x bands-in); both split into TF32 hi + lo in shared memory per 32-band slice.
// grid = (ceil(N/128), ceil(m/nt)).
template <int NC>
__global__ void __launch_bounds__(TC_THREADS, 1)
    rotate_tc_kernel(const double* __restrict__ V, long long ldv, int k, const double* __restrict__ Y, int m,
                     int nt, double* __restrict__ X, long long ldx, long long n, int* __restrict__ error) {
    extern __shared__ __align__(1024) uint32_t sm[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t bar[2];
    constexpr int NW = TC_THREADS / 32;
    constexpr int CA = TC_M * TC_KT / 32 / NW;  // core matrices of the V slice per warp (16)
    constexpr int EB = NC * TC_KT / 32 / NW;    // core matrices of the Y slice per warp
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long p0 = (long long)blockIdx.x * TC_M;
    const int j0 = blockIdx.y * nt, ncols = min(nt, m - j0);
    constexpr int a_words = TC_M * TC_KT, b_words = NC * TC_KT;
    constexpr int stage_words = 2 * a_words + 2 * b_words;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(NC));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_tf32(NC);
    // as in the Gram kernel: thread (warp, lane) owns element (row 8 rg + lane / 4,
    // k 4 kg + lane % 4) of core matrix cm = warp + 8 i; rows are points (V) or output bands (Y)
    double xa[CA], xb[EB];
    const int lr = lane >> 2, lk = lane & 3;
    auto load = [&](int k0) {
#pragma unroll
        for (int i = 0; i < CA; ++i) {
            const int cm = warp + i * NW;
            const long long p = p0 + (cm >> 3) * 8 + lr;
            const int kk = k0 + (cm & 7) * 4 + lk;
            xa[i] = (kk < k && p < n) ? __ldg(V + (long long)kk * ldv + p) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < EB; ++i) {
            const int cm = warp + i * NW;
            const int c = (cm >> 3) * 8 + lr, kk = k0 + (cm & 7) * 4 + lk;
            xb[i] = (kk < k && c < ncols) ? __ldg(Y + (long long)kk * m + j0 + c) : 0.0;
        }
    };
    load(0);
    bool ok = true;
    uint32_t phase[2] = {0, 0};
    bool pending[2] = {false, false};
    int step = 0;
    for (int k0 = 0; k0 < k; k0 += TC_KT, ++step) {
        const int st = step & 1;
        if (pending[st]) {
            if (!mbar_wait(&bar[st], phase[st])) ok = false;
            phase[st] ^= 1;
            pending[st] = false;
        }
        if (!__syncthreads_and(ok)) break;
        uint32_t* ahi = sm + st * stage_words;
        uint32_t* alo = ahi + a_words;
        uint32_t* bhi = alo + a_words;
        uint32_t* blo = bhi + b_words;
#pragma unroll
        for (int i = 0; i < CA; ++i) {
            const int cm = warp + i * NW;
            const uint32_t h = to_tf32((float)xa[i]);
            const uint32_t l = to_tf32((float)(xa[i] - (double)__uint_as_float(h)));
            const int o = (((cm & 7) * (TC_M / 8) + (cm >> 3)) << 5) + lane;
            ahi[o] = h;
            alo[o] = l;
        }
#pragma unroll
        for (int i = 0; i < EB; ++i) {
            const int cm = warp + i * NW;
            const uint32_t h = to_tf32((float)xb[i]);
            const uint32_t l = to_tf32((float)(xb[i] - (double)__uint_as_float(h)));
            const int o = (((cm & 7) * (NC / 8) + (cm >> 3)) << 5) + lane;
            bhi[o] = h;
            blo[o] = l;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t lbo_a = (TC_M / 8) * 128, lbo_b = (uint32_t)(NC / 8) * 128, sbo = 128;
            const uint32_t sa_hi = smem_u32(ahi), sa_lo = smem_u32(alo), sb_hi = smem_u32(bhi), sb_lo = smem_u32(blo);
#pragma unroll
            for (int kk = 0; kk < TC_KT / 8; ++kk) {
                const uint32_t oa = kk * 2 * lbo_a, ob = kk * 2 * lbo_b;
                const uint64_t dah = smem_desc(sa_hi + oa, lbo_a, sbo), dal = smem_desc(sa_lo + oa, lbo_a, sbo);
                const uint64_t dbh = smem_desc(sb_hi + ob, lbo_b, sbo), dbl = smem_desc(sb_lo + ob, lbo_b, sbo);
                const uint32_t first = (step == 0 && kk == 0) ? 0u : 1u;
                mma_tf32(tmem, dah, dbh, idesc, first);
                mma_tf32(tmem, dah, dbl, idesc, 1u);
                mma_tf32(tmem, dal, dbh, idesc, 1u);
            }
            mma_commit(&bar[st]);
        }
        pending[st] = true;
        if (k0 + TC_KT < k) load(k0 + TC_KT);
    }
    for (int st = 0; st < 2; ++st)
        if (pending[st]) {
            if (!mbar_wait(&bar[st], phase[st])) ok = false;
            phase[st] ^= 1;
        }
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0) atomicExch(error, 1);
    } else {
        // TMEM lane = point p0 + row; warps w and w + 4 split the columns
        const int q4 = warp & 3, half = warp >> 2;
        const long long p = p0 + q4 * 32 + lane;
        constexpr int CH = NC / (NW / 4);
        for (int c0 = half * CH; c0 < half * CH + CH; c0 += 8) {
            uint32_t v[8];
            const uint32_t addr = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (p < n)
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (c0 + q < ncols) X[(long long)(j0 + c0 + q) * ldx + p] = (double)__uint_as_float(v[q]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NC));
}

// TMA variant of the Gram tile (tuning key "tensor_core_tma"): one elected thread loads each
// 16-point K slice of the A tile (128 rows) and the B tile (NC rows) with cp.async.bulk.tensor
// (2-D maps over [rows, points], 128-byte swizzle, rows past ka/kb and points past n
// zero-filled) into a ring of S FP64 stages tracked by mbarriers with transaction counts, so
// S - 1 slices are in flight per block and no registers hold them; the warps then split each
// slice from shared memory into the TF32 hi/lo planes of one of two operand stages (the same
// K-major core-matrix layout and MMAs as gram_tc_kernel, K = 16 per slice).  With the swizzle,
// a warp's reads of 8 rows x 4 points of a slice and its 128-byte core-matrix stores are both
// free of bank conflicts.  Needs even leading dimensions and 16-byte-aligned A and B.
constexpr int TT_KT = 16;  // points per slice: one 128-byte swizzle row of FP64 per band

template <int NC>
struct TmaCfg {
    static constexpr int S = NC <= 128 ? 4 : 2;     // FP64 ring stages
    static constexpr int A_BYTES = TC_M * TT_KT * 8;  // FP64 A slice = A hi + lo planes
    static constexpr int B_BYTES = NC * TT_KT * 8;
    static constexpr int STAGE = A_BYTES + B_BYTES;
    static constexpr size_t SMEM = (size_t)STAGE * (S + 2) + 1024;
};

template <int NC>
__global__ void __launch_bounds__(TC_THREADS, 1)
    gram_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int ka, int kb,
                    long long n, long long chunk, double* __restrict__ partial, int* __restrict__ error) {
    using Cfg = TmaCfg<NC>;
    constexpr int S = Cfg::S;
    extern __shared__ uint8_t smraw[];
    uint8_t* sm = (uint8_t*)(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t mmab[2];
    constexpr int NW = TC_THREADS / 32;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_M, n0 = blockIdx.y * NC;
    const int mrows = min(TC_M, ka - m0), nrows = min(NC, kb - n0);
    const long long p0 = (long long)blockIdx.z * chunk, p1 = min(n, p0 + chunk);
    const int nslices = p1 > p0 ? (int)((p1 - p0 + TT_KT - 1) / TT_KT) : 0;
    uint8_t* fp64 = sm;                         // S stages: A slice then B slice, row-major, swizzled
    uint8_t* opnd = sm + (size_t)S * Cfg::STAGE;  // 2 stages: A hi, A lo, B hi, B lo
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(NC));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int q = 0; q < S; ++q) mbar_init(&full[q], 1);
        mbar_init(&mmab[0], 1);
        mbar_init(&mmab[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_tf32(NC);
    int issued = 0;
    auto issue = [&](int q) {  // slice q into FP64 stage q % S (thread 0)
        uint8_t* st = fp64 + (size_t)(q % S) * Cfg::STAGE;
        const uint32_t bar = smem_u32(&full[q % S]);
        const int x = (int)(p0 + (long long)q * TT_KT);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(Cfg::STAGE) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_u32(st)),
            "l"(reinterpret_cast<uint64_t>(&tmA)), "r"(x), "r"(m0), "r"(bar)
            : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_u32(st + Cfg::A_BYTES)),
            "l"(reinterpret_cast<uint64_t>(&tmB)), "r"(x), "r"(n0), "r"(bar)
            : "memory");
    };
    if (tid == 0)
        for (; issued < nslices && issued < S; ++issued) issue(issued);
    bool ok = true;
    int waited_full = 0;  // slices whose TMA this thread has waited for
    int s = 0;
    // element (row, k) of a swizzled FP64 slice: 16-byte chunk k/2 of row `row` is stored at
    // chunk (k/2) ^ (row % 8) (128-byte swizzle)
    auto fp_at = [](const uint8_t* base, int row, int k) {
        return *(const double*)(base + row * 128 + ((((k >> 1) ^ (row & 7)) << 4) | ((k & 1) << 3)));
    };
    for (; s < nslices; ++s) {
        const int fs = s % S, os = s & 1;
        if (s >= 2 && !mbar_wait(&mmab[os], (uint32_t)(((s - 2) >> 1) & 1))) ok = false;
        if (ok && !mbar_wait(&full[fs], (uint32_t)((s / S) & 1))) ok = false;
        if (ok) waited_full = s + 1;
        if (!__syncthreads_and(ok)) break;
        const uint8_t* fa = fp64 + (size_t)fs * Cfg::STAGE;
        const uint8_t* fb = fa + Cfg::A_BYTES;
        uint32_t* ahi = (uint32_t*)(opnd + (size_t)os * Cfg::STAGE);
        uint32_t* alo = ahi + TC_M * TT_KT;
        uint32_t* bhi = alo + TC_M * TT_KT;
        uint32_t* blo = bhi + NC * TT_KT;
        // core matrix cm = kc * (R/8) + rg holds rows 8 rg .. +7, points 4 kc .. +3; lane l
        // owns row 8 rg + l/4, point 4 kc + l%4, i.e. word 32 cm + l
#pragma unroll
        for (int i = 0; i < (TC_M * TT_KT / 32) / NW; ++i) {
            const int cm = warp + i * NW, kc = cm / (TC_M / 8), rg = cm % (TC_M / 8);
            const double x = fp_at(fa, rg * 8 + (lane >> 2), kc * 4 + (lane & 3));
            const uint32_t h = to_tf32((float)x);
            ahi[cm * 32 + lane] = h;
            alo[cm * 32 + lane] = to_tf32((float)(x - (double)__uint_as_float(h)));
        }
#pragma unroll
        for (int i = 0; i < (NC * TT_KT / 32) / NW; ++i) {
            const int cm = warp + i * NW, kc = cm / (NC / 8), rg = cm % (NC / 8);
            const double x = fp_at(fb, rg * 8 + (lane >> 2), kc * 4 + (lane & 3));
            const uint32_t h = to_tf32((float)x);
            bhi[cm * 32 + lane] = h;
            blo[cm * 32 + lane] = to_tf32((float)(x - (double)__uint_as_float(h)));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t lbo_a = (TC_M / 8) * 128, lbo_b = (uint32_t)(NC / 8) * 128, sbo = 128;
            const uint32_t sa_hi = smem_u32(ahi), sa_lo = smem_u32(alo), sb_hi = smem_u32(bhi), sb_lo = smem_u32(blo);
#pragma unroll
            for (int kk = 0; kk < TT_KT / 8; ++kk) {
                const uint32_t oa = kk * 2 * lbo_a, ob = kk * 2 * lbo_b;
                const uint64_t dah = smem_desc(sa_hi + oa, lbo_a, sbo), dal = smem_desc(sa_lo + oa, lbo_a, sbo);
                const uint64_t dbh = smem_desc(sb_hi + ob, lbo_b, sbo), dbl = smem_desc(sb_lo + ob, lbo_b, sbo);
                const uint32_t first = (s == 0 && kk == 0) ? 0u : 1u;
                mma_tf32(tmem, dah, dbh, idesc, first);
                mma_tf32(tmem, dah, dbl, idesc, 1u);
                mma_tf32(tmem, dal, dbh, idesc, 1u);
            }
            mma_commit(&mmab[os]);
            // every thread has split FP64 stage fs (barrier above): refill it with slice s + S
            if (issued < nslices) issue(issued++);
        }
    }
    // drain: the last two slices' MMAs, then (after a give-up) the TMA loads still in flight
    for (int q = max(0, s - 2); q < s; ++q)
        if (!mbar_wait(&mmab[q & 1], (uint32_t)((q >> 1) & 1))) ok = false;
    if (tid == 0)
        for (int q = waited_full; q < issued; ++q) mbar_wait(&full[q % S], (uint32_t)((q / S) & 1));
    ok = __syncthreads_and(ok);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    double* out = partial + (long long)blockIdx.z * ka * kb;
    if (!ok) {
        if (tid == 0) atomicExch(error, 1);
    } else if (nslices > 0) {
        const int q4 = warp & 3, half = warp >> 2;
        const int row = q4 * 32 + lane;
        constexpr int CH = NC / (NW / 4);
        for (int c0 = half * CH; c0 < half * CH + CH; c0 += 8) {
            uint32_t v[8];
            const uint32_t addr = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < mrows)
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (c0 + q < nrows) out[(long long)(m0 + row) * kb + (n0 + c0 + q)] = (double)__uint_as_float(v[q]);
        }
    } else {
        for (int e = tid; e < mrows * nrows; e += TC_THREADS)
            out[(long long)(m0 + e / nrows) * kb + (n0 + e % nrows)] = 0.0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NC));
}

// 2-D map over rows x points of a band block (row stride ld doubles), box 16 points x rows
CUtensorMap band_tensor_map(const double* base, long long ld, long long n, int rows, int box_rows) {
    CUtensorMap tm;
    const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
    const cuuint32_t box[2] = {TT_KT, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = tensor_map_encoder()(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims,
                                            strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(DFT_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return tm;
}

}  // namespace

// C (ka x kb, host, row-major) = dV * A^T B on the tensor cores (TF32 hi+lo split).
void gram_tc(dft_context* ctx, const Grid& g, const double* A, long long lda, int ka, const double* B, long long ldb,
             int kb, std::vector<double>& C) {
    C.assign((size_t)ka * kb, 0.0);
    if (ka == 0 || kb == 0) return;
    // N tile: up to 256 columns, a multiple of 16, TMEM allocation a power of two >= 32
    const int ntiles = (kb + TC_NMAX - 1) / TC_NMAX;
    const int nt = (kb + ntiles - 1) / ntiles;
    int ncols = 32;
    while (ncols < nt) ncols <<= 1;
    const int mtiles = (ka + TC_M - 1) / TC_M;
    const size_t smem = sizeof(uint32_t) * 2 * (size_t)(2 * TC_M * TC_KT + 2 * ncols * TC_KT);
    // split K so that each block accumulates <= 8192 points in FP32 and the machine is covered
    long long nch = std::max<long long>(1, (2LL * ctx->num_sms) / (mtiles * ntiles));
    nch = std::max<long long>(nch, (g.N + 8191) / 8192);
    long long chunk = (g.N + nch - 1) / nch;
    chunk = ((chunk + TC_KT - 1) / TC_KT) * TC_KT;
    nch = (g.N + chunk - 1) / chunk;
    const size_t nel = (size_t)ka * kb;
    double* partial = (double*)ws_get(ctx, WS_SMALL, sizeof(double) * (nel * nch + nel) + 64);
    double* res = partial + nel * nch;
    int* err = (int*)(res + nel);
    static bool attr = false;
    if (!attr) {
        DFT_CUDA(cudaFuncSetAttribute(gram_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        DFT_CUDA(cudaFuncSetAttribute(gram_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        DFT_CUDA(cudaFuncSetAttribute(gram_tc_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        DFT_CUDA(cudaFuncSetAttribute(gram_tc_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
    DFT_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    const bool tma = ctx->tc_tma && lda % 2 == 0 && ldb % 2 == 0 && ((uintptr_t)A & 15) == 0 &&
                     ((uintptr_t)B & 15) == 0 && tensor_map_encoder() != nullptr;
    if (tma) {
        // tiles of exactly ncols columns (the B box); rows past kb are zero-filled by the copy
        static bool tattr = false;
        if (!tattr) {
            DFT_CUDA(cudaFuncSetAttribute(gram_tma_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)TmaCfg<32>::SMEM));
            DFT_CUDA(cudaFuncSetAttribute(gram_tma_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)TmaCfg<64>::SMEM));
            DFT_CUDA(cudaFuncSetAttribute(gram_tma_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)TmaCfg<128>::SMEM));
            DFT_CUDA(cudaFuncSetAttribute(gram_tma_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)TmaCfg<256>::SMEM));
            tattr = true;
        }
        const int nt2 = (kb + ncols - 1) / ncols;
        const CUtensorMap tmA = band_tensor_map(A, lda, g.N, ka, TC_M);
        const CUtensorMap tmB = band_tensor_map(B, ldb, g.N, kb, ncols);
        const dim3 grid2(mtiles, nt2, (unsigned)nch);
        switch (ncols) {
            case 32:
                gram_tma_kernel<32><<<grid2, TC_THREADS, TmaCfg<32>::SMEM, ctx->stream>>>(tmA, tmB, ka, kb, g.N, chunk,
                                                                                         partial, err);
                break;
            case 64:
                gram_tma_kernel<64><<<grid2, TC_THREADS, TmaCfg<64>::SMEM, ctx->stream>>>(tmA, tmB, ka, kb, g.N, chunk,
                                                                                         partial, err);
                break;
            case 128:
                gram_tma_kernel<128><<<grid2, TC_THREADS, TmaCfg<128>::SMEM, ctx->stream>>>(tmA, tmB, ka, kb, g.N,
                                                                                           chunk, partial, err);
                break;
            default:
                gram_tma_kernel<256><<<grid2, TC_THREADS, TmaCfg<256>::SMEM, ctx->stream>>>(tmA, tmB, ka, kb, g.N,
                                                                                           chunk, partial, err);
                break;
        }
    }
    const dim3 grid(mtiles, ntiles, (unsigned)nch);
    const bool ring = ctx->tc_ring && ncols <= 128 && lda % 2 == 0 && ldb % 2 == 0 &&
                      ((uintptr_t)A & 15) == 0 && ((uintptr_t)B & 15) == 0;
    if (tma) {
        // launched above
    } else if (ring) {
        static bool rattr = false;
        if (!rattr) {
            DFT_CUDA(cudaFuncSetAttribute(gram_tc_ring_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)ring_smem<32>()));
            DFT_CUDA(cudaFuncSetAttribute(gram_tc_ring_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)ring_smem<64>()));
            DFT_CUDA(cudaFuncSetAttribute(gram_tc_ring_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)ring_smem<128>()));
            rattr = true;
        }
        if (ncols == 32)
            gram_tc_ring_kernel<32><<<grid, TC_THREADS, ring_smem<32>(), ctx->stream>>>(A, lda, ka, B, ldb, kb, nt, g.N,
                                                                                       chunk, partial, err);
        else if (ncols == 64)
            gram_tc_ring_kernel<64><<<grid, TC_THREADS, ring_smem<64>(), ctx->stream>>>(A, lda, ka, B, ldb, kb, nt, g.N,
                                                                                       chunk, partial, err);
        else
            gram_tc_ring_kernel<128><<<grid, TC_THREADS, ring_smem<128>(), ctx->stream>>>(A, lda, ka, B, ldb, kb, nt,
                                                                                         g.N, chunk, partial, err);
    } else switch (ncols) {
        case 32:
            gram_tc_kernel<32><<<grid, TC_THREADS, smem, ctx->stream>>>(A, lda, ka, B, ldb, kb, nt, g.N, chunk,
                                                                        partial, err);
            break;
        case 64:
            gram_tc_kernel<64><<<grid, TC_THREADS, smem, ctx->stream>>>(A, lda, ka, B, ldb, kb, nt, g.N, chunk,
                                                                        partial, err);
            break;
        case 128:
            gram_tc_kernel<128><<<grid, TC_THREADS, smem, ctx->stream>>>(A, lda, ka, B, ldb, kb, nt, g.N, chunk,
                                                                         partial, err);
            break;
        default:
            gram_tc_kernel<256><<<grid, TC_THREADS, smem, ctx->stream>>>(A, lda, ka, B, ldb, kb, nt, g.N, chunk,
                                                                         partial, err);
            break;
    }
    DFT_LAUNCH_CHECK();
    const int rb = (int)std::min<size_t>((nel + 7) / 8, 4096);
    gram_tc_reduce_kernel<<<rb, 256, 0, ctx->stream>>>((int)nch, (int)nel, partial, g.dV, res);
    DFT_LAUNCH_CHECK();
    count_launch(ctx, 2);
    ctx->tc_launches += 1;
    double* h = pinned(ctx, nel + 1);
    DFT_CUDA(cudaMemcpyAsync(h, res, sizeof(double) * nel, cudaMemcpyDeviceToHost, ctx->stream));
    DFT_CUDA(cudaMemcpyAsync(h + nel, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    if (*(int*)(h + nel)) fail(DFT_CUDA_ERROR, "tensor-core Gram: mbarrier wait timed out");
    std::copy(h, h + nel, C.begin());
}

// X (m bands, leading dimension ldx) = V (k bands, ldv) * Y (k x m, host row-major) on the
// tensor cores (TF32 hi+lo split, FP32 accumulation over k <= 4096 bands).
void rotate_tc(dft_context* ctx, const Grid& g, const double* V, long long ldv, int k, const std::vector<double>& Y,
               int m, double* X, long long ldx) {
    if (m == 0) return;
    if (k == 0) {
        for (int j = 0; j < m; ++j)
            DFT_CUDA(cudaMemsetAsync(X + (long long)j * ldx, 0, sizeof(double) * (size_t)g.N, ctx->stream));
        return;
    }
    if (k > 4096) fail(DFT_INVALID_ARGUMENT, "rotation over more than 4096 bands");
    const int ntiles = (m + TC_NMAX - 1) / TC_NMAX;
    const int nt = (m + ntiles - 1) / ntiles;
    int ncols = 32;
    while (ncols < nt) ncols <<= 1;
    const size_t smem = sizeof(uint32_t) * 2 * (size_t)(2 * TC_M * TC_KT + 2 * ncols * TC_KT);
    double* dy = (double*)ws_get(ctx, WS_TMP, sizeof(double) * (size_t)k * m);
    int* err = (int*)ws_get(ctx, WS_TMP2, 64);
    DFT_CUDA(cudaMemcpyAsync(dy, Y.data(), sizeof(double) * (size_t)k * m, cudaMemcpyHostToDevice, ctx->stream));
    DFT_CUDA(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
    static bool attr = false;
    if (!attr) {
        DFT_CUDA(cudaFuncSetAttribute(rotate_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        DFT_CUDA(cudaFuncSetAttribute(rotate_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        DFT_CUDA(cudaFuncSetAttribute(rotate_tc_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        DFT_CUDA(cudaFuncSetAttribute(rotate_tc_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
    const dim3 grid((unsigned)((g.N + TC_M - 1) / TC_M), (unsigned)ntiles);
    switch (ncols) {
        case 32:
            rotate_tc_kernel<32><<<grid, TC_THREADS, smem, ctx->stream>>>(V, ldv, k, dy, m, nt, X, ldx, g.N, err);
            break;
        case 64:
            rotate_tc_kernel<64><<<grid, TC_THREADS, smem, ctx->stream>>>(V, ldv, k, dy, m, nt, X, ldx, g.N, err);
            break;
        case 128:
            rotate_tc_kernel<128><<<grid, TC_THREADS, smem, ctx->stream>>>(V, ldv, k, dy, m, nt, X, ldx, g.N, err);
            break;
        default:
            rotate_tc_kernel<256><<<grid, TC_THREADS, smem, ctx->stream>>>(V, ldv, k, dy, m, nt, X, ldx, g.N, err);
            break;
    }
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    ctx->tc_launches += 1;
    int* h = (int*)pinned(ctx, 1);
    DFT_CUDA(cudaMemcpyAsync(h, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);  // also keeps Y alive until its copy has run
    if (*h) fail(DFT_CUDA_ERROR, "tensor-core rotation: mbarrier wait timed out");
}

}  // namespace dftb
