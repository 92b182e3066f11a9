// Shared host/device plumbing for the dft_b200 kernels: status handling, the context,
// the device grid descriptor and deterministic block reductions.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdarg>
#include <map>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/dft_b200.h"

namespace dftb {

// ---------------------------------------------------------------- status -----
// Internal code throws dftb::Error; the C ABI converts it into a status + message.
struct Error : std::runtime_error {
    dft_status_t status;
    Error(dft_status_t s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(dft_status_t s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Error(s, buf);
}

#define DFT_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            ::dftb::fail(DFT_CUDA_ERROR, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),    \
                         __FILE__, __LINE__);                                                       \
    } while (0)

#define DFT_LAUNCH_CHECK() DFT_CUDA(cudaGetLastError())

// ---------------------------------------------------------------- grid -------
// Device-side grid descriptor.  Spacing and inverse squares are derived on the host in
// the reference's operation order (CartesianGrid.cpp:45-47, KohnShamHamiltonianMolecule.cpp:45-55).
struct Grid {
    int nx, ny, nz;
    long long N;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double dx, dy, dz;
    double ix2, iy2, iz2;  // 1/(d*d)
    double dV;             // dx*dy*dz
};

inline Grid make_grid(const dft_grid* g) {
    if (!g) fail(DFT_INVALID_ARGUMENT, "grid is NULL");
    if (g->nx < 2 || g->ny < 2 || g->nz < 2)
        fail(DFT_INVALID_ARGUMENT, "CartesianGrid requires at least two points per dimension.");
    if (g->xmax <= g->xmin || g->ymax <= g->ymin || g->zmax <= g->zmin)
        fail(DFT_INVALID_ARGUMENT, "CartesianGrid requires valid spatial bounds.");
    if (g->nx > (1 << 20) || g->ny > (1 << 20) || g->nz > (1 << 20))
        fail(DFT_INVALID_ARGUMENT, "grid dimension too large");
    // stencil kernels use 32-bit offsets within one field
    if ((long long)g->nx * g->ny * g->nz >= (1LL << 31) - 1)
        fail(DFT_INVALID_ARGUMENT, "grids of 2^31 points or more are not supported");
    Grid d;
    d.nx = (int)g->nx;
    d.ny = (int)g->ny;
    d.nz = (int)g->nz;
    d.N = (long long)g->nx * g->ny * g->nz;
    d.xmin = g->xmin; d.xmax = g->xmax;
    d.ymin = g->ymin; d.ymax = g->ymax;
    d.zmin = g->zmin; d.zmax = g->zmax;
    d.dx = (g->xmax - g->xmin) / (double)(g->nx - 1);
    d.dy = (g->ymax - g->ymin) / (double)(g->ny - 1);
    d.dz = (g->zmax - g->zmin) / (double)(g->nz - 1);
    d.ix2 = 1.0 / (d.dx * d.dx);
    d.iy2 = 1.0 / (d.dy * d.dy);
    d.iz2 = 1.0 / (d.dz * d.dz);
    d.dV = d.dx * d.dy * d.dz;
    return d;
}

// ---------------------------------------------------------------- context ----
// Device workspace that grows on demand and is reused across calls.
struct Workspace {
    void* ptr = nullptr;
    size_t bytes = 0;
};

}  // namespace dftb

// captured multigrid cycles (poisson_start.cu), keyed by grid and buffer addresses
using MGGraphKey = std::array<long long, 6>;
struct MGGraph {
    cudaGraphExec_t exec;
    long long launches;  // kernels per replay
};

// One element's radial atom, kept for the superposed-atoms start: total density and the
// alpha shells' radial functions on the radial grid (device), and each shell's (n, l).
struct RadialTable {
    double* dens = nullptr;
    double* orbs = nullptr;
    std::vector<std::array<int, 2>> shells;
};

struct dft_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    long long tc_launches = 0;  // of which tensor-core (tcgen05) eigensolver products
    int num_sms = 148;
    // tuning knobs (dft_context_set_tuning)
    int jacobi_sweeps_per_launch = 0;  // 0 = auto, 1 = one sweep per launch, 2/4/8 = temporal blocking
    int net_tensor_cores = 1;          // network convolutions on tcgen05 (1) or FP32 CUDA cores (0)
    int hpsi_bands_per_thread = 0;     // H psi bands per thread: 0 = auto, 1, 2 or 4
    int hpsi_variant = 0;              // H psi: 0 = neighbours through L1, 1 = shared-memory plane tile,
                                       // 2 = TMA plane ring (where eligible, else 0)
    int* dev_status = nullptr;         // device word set by kernels whose bounded waits gave up
    int hpsi_zchunk = 0;               // H psi march length per block (0 = auto)
    int ortho_adaptive = 1;            // FP64 orthonormalisation: skip the second pass when safe (1)
    int mg_fused_restrict = 1;         // multigrid: one-pass 3-D restriction on fine grids <= 64^3 (1)
    int mg_coarsest_sor = 1;           // multigrid: red-black SOR coarsest solve (1) or Jacobi sweeps (0)
    int tc_ring = 0;                   // tensor-core Gram: cp.async ring variant (1) or register staging (0)
    int tc_tma = 0;                    // tensor-core Gram: TMA-fed FP64 ring (1; before tc_ring)
    long long grid_barrier_poll_limit = 0;  // persistent Jacobi barrier polls before giving up (0 = 2^24)
    // autotuner choices per grid (nx, ny, nz) -> {H psi bands per thread, Jacobi sweeps per launch},
    // used where the corresponding knob is 0 (auto)
    // {H psi bands per thread (or per block for the TMA ring), Jacobi sweeps per launch, H psi
    // variant, H psi z-march length (0 = auto)}
    std::map<std::array<long long, 3>, std::array<int, 4>> tuned;
    int multigrid_graphs = 1;                 // replay captured multigrid cycles (1) or launch directly (0)
    std::map<MGGraphKey, MGGraph> mg_graphs;  // the captured cycles
    int radial_pivot_exp = -14;        // radial inverse iteration: |pivot| < 10^exp is singular
    // named scratch buffers (reductions, Jacobi ping-pong, XC intermediates, Davidson)
    dftb::Workspace ws[32];
    double* host_pinned = nullptr;  // small pinned staging area for scalars
    size_t host_pinned_bytes = 0;
    void* gram_ticket = nullptr;    // block counter of the one-launch narrow Gram product
    // device buffers an SCF released, kept for the next SCF of the same sizes (bytes -> pointer):
    // repeated cudaMalloc/cudaFree of the SCF state stalled single solves by up to 0.5 s
    std::multimap<size_t, void*> buf_pool;
    size_t buf_pool_bytes = 0;
    // radial atoms already solved for the superposed-atoms start: {Z, kind, points, rmax bits}
    std::map<std::array<long long, 4>, RadialTable> radial_tables;
};

namespace dftb {

enum WsSlot {
    WS_REDUCE = 0,   // block partial sums
    WS_CTRL = 1,     // small control words (Jacobi state, flags)
    WS_JACOBI = 2,   // Jacobi ping-pong buffer
    WS_XC = 3,       // XC intermediates (4N)
    WS_DAV0 = 4,     // Davidson workspaces
    WS_DAV1 = 5,
    WS_DAV2 = 6,
    WS_DAV3 = 7,
    WS_DAV4 = 8,
    WS_DAV5 = 9,
    WS_SMALL = 10,   // small dense matrices on device
    WS_SCF0 = 11,
    WS_SCF1 = 12,
    WS_RADIAL = 13,
    WS_TMP = 14,
    WS_TMP2 = 15,
    WS_DAV6 = 16,    // Davidson per-band scalars on device
    WS_SCF2 = 17,
    WS_SCF3 = 18,
    WS_PG0 = 19,     // coarse-grid Poisson start (neural.cu)
    WS_PG1 = 20,
    WS_PG2 = 21,
    WS_PG3 = 22,
    WS_PG4 = 23,
    WS_TMP3 = 24,    // superposition start tables (atomic_start.cu)
    WS_NUM = 25,     // slots in use (dft_context::ws has room for 32)
};

void* ws_get(dft_context* ctx, int slot, size_t bytes);
double* pinned(dft_context* ctx, size_t count);
void sync(dft_context* ctx);

// Counts a launch on the context (bench reports how many kernels ran in a timed region).
inline void count_launch(dft_context* ctx, long long n = 1) { ctx->launches += n; }

// ---------------------------------------------------------------- device helpers --
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum in a fixed order (deterministic for a fixed launch shape).
// `sh` must hold blockDim/32 doubles.  Result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < nw; ++w) s += sh[w];
    __syncthreads();
    return s;
}

}  // namespace dftb
