// Finite-difference gradients of the XC path (device, inline): shared by the whole-grid XC
// kernels (grid_ops.cu) and the z-slab XC energy (zslab.cu), so both compute the same values.
#pragma once

#include "common.cuh"

namespace dftb {

// calculateCartesianDerivative, reference ExchangeCorrelationMolecule.cpp:11-170
__device__ __forceinline__ double dderiv(const Grid& g, const double* __restrict__ f, long long p, int i, int j, int k,
                                         int dir) {
    if (dir == 0) {
        if (i == 0) return (f[p + 1] - f[p]) / g.dx;
        if (i == g.nx - 1) return (f[p] - f[p - 1]) / g.dx;
        return (f[p + 1] - f[p - 1]) / (2.0 * g.dx);
    }
    if (dir == 1) {
        const long long s = g.nx;
        if (j == 0) return (f[p + s] - f[p]) / g.dy;
        if (j == g.ny - 1) return (f[p] - f[p - s]) / g.dy;
        return (f[p + s] - f[p - s]) / (2.0 * g.dy);
    }
    const long long s = (long long)g.nx * g.ny;
    if (k == 0) return (f[p + s] - f[p]) / g.dz;
    if (k == g.nz - 1) return (f[p] - f[p - s]) / g.dz;
    return (f[p + s] - f[p - s]) / (2.0 * g.dz);
}

__device__ __forceinline__ double gradmag(const Grid& g, const double* __restrict__ f, long long p, int i, int j, int k) {
    const double gx = dderiv(g, f, p, i, j, k, 0), gy = dderiv(g, f, p, i, j, k, 1), gz = dderiv(g, f, p, i, j, k, 2);
    return sqrt(gx * gx + gy * gy + gz * gz);
}

}  // namespace dftb
