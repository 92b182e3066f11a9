// Batched radial-atom SCF: every run (atom x functional) is one thread block of a single
// persistent launch, iterating its own SCF loop to convergence (reference
// solveSelfConsistentField, SelfConsistentField.cpp:539-786) while the other runs proceed
// independently on other SMs.  Per-run arrays (2000 points each) stay in L2.
//
// Inside a block the work that the reference does point by point runs across threads, and
// each (n,l,spin) orbital is owned by one warp:
//  * eigenvalue: the reference's Sturm bisection (EigenvalueSolver.cpp:94-221), made
//    parallel without changing its result: 31 lanes evaluate the Sturm counts at the
//    midpoints of the next five bisection levels for every possible path (a depth-5
//    speculation tree); the warp then walks the tree with the real counts.  The visited
//    midpoints, hence the final interval, are exactly the sequential ones.
//  * eigenvector: inverse iteration with the shifted Thomas factorisation computed once
//    per orbital (identical to refactoring every solve, NumericalMethods.cpp:85-139).
//  * every sum the reference takes sequentially (norms, dots, trapezoid prefix sums,
//    energies) is taken sequentially by one lane, so rounding follows the reference.
// The file is compiled without FMA contraction.  Remaining differences from the reference
// come from the device's transcendental functions (a few ulp) in XC and the start vectors.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "ops.h"
#include "xc_device.cuh"

namespace dftb {

namespace {

constexpr int RT = 512;        // threads per run
constexpr int RW = RT / 32;    // warps per run
constexpr int MAXORB = 16;     // occupied (n,l,spin) orbitals per run
constexpr double EPS = 1.0e-14;

struct RunSpec {
    int Z, kind, norb;
    double pivot_eps;  // |pivot| below this is singular (EPS unless tuned)
    int n[MAXORB], l[MAXORB], spin[MAXORB], el[MAXORB], idx[MAXORB];
};

// per-run global arrays, each n doubles
enum {
    A_DA = 0, A_DB, A_VA, A_VB, A_VH, A_OA, A_OB, A_RD, A_OD, A_T1, A_T2, A_T3, A_T4, A_ENC, A_OUT,
    A_COUNT
};
// per-orbital arrays
enum { O_U = 0, O_DIAG, O_DW, O_F, O_NX, O_COUNT };

__device__ __forceinline__ double eps_guard(double v) { return fabs(v) < EPS ? copysign(EPS, v == 0.0 ? 1.0 : v) : v; }

// countEigenvaluesBelow (EigenvalueSolver.cpp:13-92); off-diagonals all equal `off`
__device__ long sturm_count(int n, const double* __restrict__ diag, double oo, double E) {
    long c = 0;
    double prev = diag[0] - E;
    if (prev < 0.0) ++c;
    prev = eps_guard(prev);
    for (int i = 1; i < n; ++i) {
        const double piv = (diag[i] - E) - oo / eps_guard(prev);
        if (piv < 0.0) ++c;
        prev = eps_guard(piv);
    }
    return c;
}

__device__ __forceinline__ double shfl_d(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }

// warp-wide: the k-th eigenvalue of the radial Hamiltonian in [lo, hi] (findEigenvalue)
__device__ bool find_eigenvalue(int n, const double* __restrict__ diag, double oo, long index, double lo, double hi,
                                double& out) {
    const int lane = threadIdx.x & 31;
    long lc = 0, hc = 0;
    {
        const long c = (lane < 2) ? sturm_count(n, diag, oo, lane == 0 ? lo : hi) : 0;
        lc = __shfl_sync(0xffffffffu, c, 0);
        hc = __shfl_sync(0xffffffffu, c, 1);
    }
    double w = hi - lo;
    for (int e = 0; e < 100; ++e) {
        if (lc <= index && index < hc) break;
        w *= 2.0;
        const bool mlo = lc > index, mhi = hc <= index;
        if (mlo) lo -= w;
        if (mhi) hi += w;
        const long c = (lane == 0 && mlo) ? sturm_count(n, diag, oo, lo) : ((lane == 1 && mhi) ? sturm_count(n, diag, oo, hi) : 0);
        const long c0 = __shfl_sync(0xffffffffu, c, 0), c1 = __shfl_sync(0xffffffffu, c, 1);
        if (mlo) lc = c0;
        if (mhi) hc = c1;
    }
    if (lc > index || index >= hc) return false;
    int iter = 0;
    bool done = false;
    while (!done && iter < 300) {
        // node t of the speculation tree: replay its path from (lo, hi)
        double nmid = 0.0;
        long ncount = 0;
        if (lane < 31) {
            int path[5], depth = 0;
            for (int t = lane; t > 0; t = (t - 1) >> 1) path[depth++] = (t & 1);  // 1 = left child (count <= index)
            double a = lo, b = hi;
            for (int s = depth - 1; s >= 0; --s) {
                const double m = 0.5 * (a + b);
                if (path[s]) a = m;
                else b = m;
            }
            nmid = 0.5 * (a + b);
            ncount = sturm_count(n, diag, oo, nmid);
        }
        int t = 0;
        for (int level = 0; level < 5 && !done && iter < 300; ++level) {
            const double mid = shfl_d(nmid, t);
            const long c = __shfl_sync(0xffffffffu, ncount, t);
            if (c <= index) {
                lo = mid;
                t = 2 * t + 1;
            } else {
                hi = mid;
                t = 2 * t + 2;
            }
            ++iter;
            const double tol = 1.0e-13 * fmax(1.0, fmax(fabs(lo), fabs(hi)));
            if (hi - lo <= tol) done = true;
        }
    }
    out = 0.5 * (lo + hi);
    return true;
}

// sequential sum_i a_i*b_i in the reference order (lane-0 helper)
__device__ double seq_dot(int n, const double* a, const double* b) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

struct Scal {
    double mixing, prevE, prevD, E[5], effd, resid;
    double dsum[6];
    double Tpart[MAXORB];
    double respart[MAXORB];
    double ee, eh, exc;
    int conv, status, iter, err_orb;
};

__global__ void __launch_bounds__(RT, 1)
    radial_scf_kernel(const RunSpec* __restrict__ specs, int npts, double rmax, double* __restrict__ ws,
                      long long per_run, dft_atom_result* __restrict__ out) {
    extern __shared__ double r[];
    __shared__ Scal S;
    const RunSpec& sp = specs[blockIdx.x];
    const int n = npts;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double* base = ws + (long long)blockIdx.x * per_run;
    auto arr = [&](int a) { return base + (long long)a * n; };
    auto orb = [&](int q, int a) { return base + (long long)(A_COUNT + q * O_COUNT + a) * n; };
    const double h = rmax / (double)(n + 1);
    for (int i = tid; i < n; i += RT) r[i] = (double)(i + 1) * h;  // RadialGrid.cpp:16-20
    __syncthreads();
    const double dr = r[1] - r[0];
    const double idr2 = 1.0 / (dr * dr);
    const double off = -0.5 * idr2;
    const double oo = off * off;
    const double fourpi = 4.0 * xcf::PI;
    const int Z = sp.Z, kind = sp.kind, norb = sp.norb;
    double *da = arr(A_DA), *db = arr(A_DB), *va = arr(A_VA), *vb = arr(A_VB), *vh = arr(A_VH);
    double *oa = arr(A_OA), *ob = arr(A_OB), *rd = arr(A_RD), *od = arr(A_OD);
    double *t1 = arr(A_T1), *t2 = arr(A_T2), *t3 = arr(A_T3), *t4 = arr(A_T4), *enc = arr(A_ENC);
    if (tid == 0) {
        S.mixing = 0.25;
        S.prevE = INFINITY;
        S.prevD = INFINITY;
        S.conv = 0;
        S.status = 0;
        S.iter = 0;
        S.err_orb = -1;
        for (int q = 0; q < 5; ++q) S.E[q] = 0.0;
        S.effd = 0.0;
        S.resid = 0.0;
    }
    __syncthreads();

    // ---- hydrogenic start orbitals and densities (SelfConsistentField.cpp:207-339) ------------
    for (int q = warp; q < norb; q += RW) {
        double* u = orb(q, O_U);
        const double ex = fmax(0.15, (double)Z / ((double)sp.n[q] * (double)sp.n[q]));
        for (int i = lane; i < n; i += 32) u[i] = pow(r[i], (double)(sp.l[q] + 1)) * exp(-ex * r[i]);
        __syncwarp();
        double nn = 0.0;
        if (lane == 0) nn = sqrt(dr * seq_dot(n, u, u));
        nn = shfl_d(nn, 0);
        if (nn < EPS) {
            if (lane == 0) { S.status = DFT_NOT_CONVERGED; S.err_orb = q; }
        } else {
            for (int i = lane; i < n; i += 32) u[i] /= nn;
        }
        __syncwarp();
    }
    __syncthreads();
    // calculateSpinDensity (ElectronDensity.cpp:8-56): orbital order, electrons*u*u/(4 pi r r)
    auto spin_densities = [&](double* a, double* b) {
        for (int i = tid; i < n; i += RT) {
            double sa = 0.0, sb = 0.0;
            const double w = fourpi * r[i] * r[i];
            for (int q = 0; q < norb; ++q) {
                const double u = orb(q, O_U)[i];
                const double v = (double)sp.el[q] * u * u / w;
                if (sp.spin[q] == 0) sa += v;
                else sb += v;
            }
            a[i] = sa;
            b[i] = sb;
        }
    };
    spin_densities(da, db);
    __syncthreads();

    // radial Hartree (HartreePotential.cpp:8-86): trapezoid terms in parallel, prefix sums in order
    auto hartree = [&](const double* rho, double* v) {
        for (int i = tid; i < n; i += RT) {
            if (i >= 1) t1[i] = 0.5 * (fourpi * r[i - 1] * r[i - 1] * rho[i - 1] + fourpi * r[i] * r[i] * rho[i]) * dr;
            if (i + 1 < n) t2[i] = 0.5 * (fourpi * r[i] * rho[i] + fourpi * r[i + 1] * rho[i + 1]) * dr;
        }
        __syncthreads();
        if (tid == 0) {
            enc[0] = 0.0;
            for (int i = 1; i < n; ++i) enc[i] = enc[i - 1] + t1[i];
        } else if (tid == 32) {
            t3[n - 1] = 0.0;
            for (int i = n - 2; i >= 0; --i) t3[i] = t3[i + 1] + t2[i];
        }
        __syncthreads();
        for (int i = tid; i < n; i += RT) v[i] = enc[i] / r[i] + t3[i];
        __syncthreads();
    };
    // calculateRadialGradient (ExchangeCorrelation.cpp:10-51)
    auto rgrad = [&](const double* f, int i) -> double {
        if (i == 0) return (f[1] - f[0]) / (r[1] - r[0]);
        if (i == n - 1) return (f[n - 1] - f[n - 2]) / (r[n - 1] - r[n - 2]);
        return (f[i + 1] - f[i - 1]) / (r[i + 1] - r[i - 1]);
    };
    // calculateRadialDivergence (:53-150)
    auto rdiv = [&](const double* c, int i) -> double {
        if (r[i] == 0.0) return 0.0;
        if (i == 0) return ((r[1] * r[1] * c[1] - r[0] * r[0] * c[0]) / (r[1] - r[0])) / (r[0] * r[0]);
        if (i == n - 1)
            return ((r[n - 1] * r[n - 1] * c[n - 1] - r[n - 2] * r[n - 2] * c[n - 2]) / (r[n - 1] - r[n - 2])) /
                   (r[n - 1] * r[n - 1]);
        return ((r[i + 1] * r[i + 1] * c[i + 1] - r[i - 1] * r[i - 1] * c[i - 1]) / (r[i + 1] - r[i - 1])) / (r[i] * r[i]);
    };
    auto evaluate = [&](int i, const double* a, const double* b) {
        return kind == 1 ? xcf::pbe96(a[i], b[i], rgrad(a, i), rgrad(b, i)) : xcf::pz81(a[i], b[i]);
    };

    for (int it = 1; it <= 250; ++it) {
        if (S.status) break;
        // ---- buildEffectivePotentials (:341-412) ------------------------------------------
        for (int i = tid; i < n; i += RT) rd[i] = da[i] + db[i];
        __syncthreads();
        hartree(rd, vh);
        for (int i = tid; i < n; i += RT) {
            const xcf::Result x = evaluate(i, da, db);
            t1[i] = x.va;  // d f / d n_alpha
            t2[i] = x.ca;
            t3[i] = x.vb;
            t4[i] = x.cb;
        }
        __syncthreads();
        for (int i = tid; i < n; i += RT) {
            const bool floor = da[i] + db[i] <= xcf::RHO_FLOOR;
            const double xa = floor ? 0.0 : (r[i] == 0.0 ? t1[i] : t1[i] - rdiv(t2, i));
            const double xb = floor ? 0.0 : (r[i] == 0.0 ? t3[i] : t3[i] - rdiv(t4, i));
            const double nuc = -(double)Z / r[i];
            va[i] = xa + (nuc + vh[i]);
            vb[i] = xb + (nuc + vh[i]);
        }
        __syncthreads();
        // ---- orbitals: one warp per (n,l,spin), index counts same-spin states per l (:28-77) --
        for (int q = warp; q < norb; q += RW) {
            const double* V = sp.spin[q] == 0 ? va : vb;
            double* diag = orb(q, O_DIAG);
            const double cc = 0.5 * (double)(sp.l[q] * (sp.l[q] + 1));
            double mn = INFINITY, mx = -INFINITY;
            for (int i = lane; i < n; i += 32) {
                const double d = idr2 + cc / (r[i] * r[i]) + V[i];  // KohnShamHamiltonian.cpp:78-86
                diag[i] = d;
                mn = fmin(mn, d);
                mx = fmax(mx, d);
            }
            for (int o = 16; o > 0; o >>= 1) {
                mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            }
            __syncwarp();
            double E = 0.0;
            if (!find_eigenvalue(n, diag, oo, sp.idx[q], mn - 10.0, mx + 10.0, E)) {
                if (lane == 0) { S.status = DFT_NOT_CONVERGED; S.err_orb = q; }
                continue;
            }
            // ---- solveEigenvector (:223-321) --------------------------------------------
            double *u = orb(q, O_U), *dw = orb(q, O_DW), *f = orb(q, O_F), *nx = orb(q, O_NX);
            for (int i = lane; i < n; i += 32) u[i] = sin((double)(i + 1));
            __syncwarp();
            double nn = 0.0;
            if (lane == 0) nn = sqrt(seq_dot(n, u, u));
            nn = shfl_d(nn, 0);
            for (int i = lane; i < n; i += 32) u[i] /= nn;
            const double shift = E + 1.0e-10 * fmax(1.0, fabs(E));
            int bad = 0;
            if (lane == 0) {
                dw[0] = diag[0] - shift;
                for (int i = 1; i < n && !bad; ++i) {
                    if (fabs(dw[i - 1]) < sp.pivot_eps) bad = 1;
                    const double fac = off / dw[i - 1];
                    f[i] = fac;
                    dw[i] = (diag[i] - shift) - fac * off;
                }
                if (fabs(dw[n - 1]) < sp.pivot_eps) bad = 1;
            }
            bad = __shfl_sync(0xffffffffu, bad, 0);
            if (bad) {
                if (lane == 0) { S.status = DFT_SINGULAR; S.err_orb = q; }
                continue;
            }
            __syncwarp();
            for (int ii = 0; ii < 1000; ++ii) {
                double m = 0.0;
                if (lane == 0) {
                    for (int i = 0; i < n; ++i) nx[i] = u[i];
                    for (int i = 1; i < n; ++i) nx[i] -= f[i] * nx[i - 1];
                    nx[n - 1] /= dw[n - 1];
                    for (int i = n - 2; i >= 0; --i) nx[i] = (nx[i] - off * nx[i + 1]) / dw[i];
                    m = sqrt(seq_dot(n, nx, nx));
                }
                m = shfl_d(m, 0);
                __syncwarp();
                if (m < EPS) {
                    if (lane == 0) { S.status = DFT_NOT_CONVERGED; S.err_orb = q; }
                    break;
                }
                for (int i = lane; i < n; i += 32) nx[i] /= m;
                __syncwarp();
                double sd = 0.0;
                if (lane == 0) sd = seq_dot(n, u, nx);
                sd = shfl_d(sd, 0);
                double md = 0.0;
                for (int i = lane; i < n; i += 32) {
                    const double v = sd < 0.0 ? -nx[i] : nx[i];
                    md = fmax(md, fabs(u[i] - v));
                    u[i] = v;
                }
                for (int o = 16; o > 0; o >>= 1) md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
                __syncwarp();
                if (md < 1.0e-12) break;
            }
            // normalizeVector(u, r[1]-r[0]) (NumericalMethods.cpp:34-61)
            double un = 0.0;
            if (lane == 0) un = sqrt(dr * seq_dot(n, u, u));
            un = shfl_d(un, 0);
            for (int i = lane; i < n; i += 32) u[i] /= un;
            if (lane == 0) out[blockIdx.x].eigenvalues[q] = E;
            __syncwarp();
        }
        __syncthreads();
        if (S.status) break;
        // ---- output densities, V_H(out), energies (:620-680, TotalEnergy.cpp) ------------
        spin_densities(oa, ob);
        __syncthreads();
        for (int i = tid; i < n; i += RT) od[i] = oa[i] + ob[i];
        __syncthreads();
        hartree(od, vh);
        // per-orbital kinetic energy and KS residual (TotalEnergy.cpp:10-101, SelfConsistentField.cpp:110-205)
        for (int q = warp; q < norb; q += RW) {
            if (lane == 0) {
                const double* u = orb(q, O_U);
                const double* V = sp.spin[q] == 0 ? va : vb;
                const double cc = 0.5 * (double)(sp.l[q] * (sp.l[q] + 1));
                const double E = out[blockIdx.x].eigenvalues[q];
                double oe = 0.0, s2 = 0.0;
                for (int i = 0; i < n; ++i) {
                    double ap = (idr2 + cc / (r[i] * r[i])) * u[i];
                    if (i > 0) ap += off * u[i - 1];
                    if (i + 1 < n) ap += off * u[i + 1];
                    oe += u[i] * ap;
                    double v = (idr2 + cc / (r[i] * r[i]) + V[i]) * u[i];
                    if (i > 0) v += off * u[i - 1];
                    if (i + 1 < n) v += off * u[i + 1];
                    const double rr = v - E * u[i];
                    s2 += rr * rr;
                }
                S.Tpart[q] = (double)sp.el[q] * oe * dr;
                S.respart[q] = sqrt(s2 * dr);
            }
        }
        // XC energy integrand (ExchangeCorrelation.cpp:276-371)
        for (int i = tid; i < n; i += RT) {
            const double dn = oa[i] + ob[i];
            double e = 0.0;
            if (dn > xcf::RHO_FLOOR) e = evaluate(i, oa, ob).eps;
            t4[i] = fourpi * r[i] * r[i] * dn * e;
        }
        __syncthreads();
        // sequential sums, one thread each
        if (tid == 0) {  // external energy (TotalEnergy.cpp:103-168)
            double e = 0.0;
            for (int i = 0; i < n; ++i) {
                const double in = -(double)Z * 4.0 * xcf::PI * r[i] * od[i];
                e += (i == 0 || i == n - 1) ? 0.5 * in : in;
            }
            S.ee = e * dr;
        } else if (tid == 32) {  // Hartree energy (HartreePotential.cpp:88-137)
            double e = 0.0;
            for (int i = 0; i < n; ++i) {
                const double in = fourpi * r[i] * r[i] * od[i] * vh[i];
                e += (i == 0 || i == n - 1) ? 0.5 * in : in;
            }
            S.eh = 0.5 * e * dr;
        } else if (tid == 64) {
            double e = 0.0;
            for (int i = 0; i < n; ++i) e += (i == 0 || i == n - 1) ? 0.5 * t4[i] : t4[i];
            S.exc = e * dr;
        } else if (tid == 96 || tid == 128 || tid == 160) {  // density differences (:414-485)
            const int w = (tid - 96) / 32;
            const double* o = w == 0 ? rd : (w == 1 ? da : db);
            const double* nw = w == 0 ? od : (w == 1 ? oa : ob);
            double d2 = 0.0, n2 = 0.0;
            for (int i = 0; i < n; ++i) {
                const double wt = 4.0 * xcf::PI * r[i] * r[i];
                const double d = nw[i] - o[i];
                d2 += d * d * wt;
                n2 += nw[i] * nw[i] * wt;
            }
            const double dn = sqrt(d2 * dr), nn = sqrt(n2 * dr);
            S.dsum[w] = nn <= EPS ? dn : dn / nn;
        }
        __syncthreads();
        if (tid == 0) {
            double T = 0.0, res = 0.0;
            for (int q = 0; q < norb; ++q) {
                T += S.Tpart[q];
                res = fmax(res, S.respart[q]);
            }
            S.E[0] = T;
            S.E[1] = S.ee;
            S.E[2] = S.eh;
            S.E[3] = S.exc;
            S.E[4] = T + S.ee + S.eh + S.exc;
            S.effd = fmax(S.dsum[0], fmax(S.dsum[1], S.dsum[2]));
            S.resid = res;
            S.iter = it;
            const double dE = isfinite(S.prevE) ? fabs(S.E[4] - S.prevE) : INFINITY;
            S.conv = (S.effd < 1.0e-9 && dE < 1.0e-11 && res < 1.0e-7) ? 1 : 0;
            if (!S.conv) {
                if (isfinite(S.prevD)) {
                    if (S.effd > S.prevD * 1.05) S.mixing = fmax(0.10, S.mixing * 0.50);
                    else if (S.effd < S.prevD) S.mixing = fmin(0.50, S.mixing * 1.10);
                }
                S.prevD = S.effd;
                S.prevE = S.E[4];
            }
        }
        __syncthreads();
        if (S.conv) break;
        // mixDensity with the updated factor (SelfConsistentField.cpp:514-535, :766-776)
        const double m = S.mixing;
        for (int i = tid; i < n; i += RT) {
            da[i] = (1.0 - m) * da[i] + m * oa[i];
            db[i] = (1.0 - m) * db[i] + m * ob[i];
        }
        __syncthreads();
    }
    if (tid == 0) {
        dft_atom_result& o = out[blockIdx.x];
        o.Z = Z;
        o.kind = kind;
        o.kinetic = S.E[0];
        o.external = S.E[1];
        o.hartree = S.E[2];
        o.exchange_correlation = S.E[3];
        o.total = S.E[4];
        o.iterations = S.iter;
        o.converged = S.conv;
        o.density_difference = S.effd;
        o.max_ks_residual = S.resid;
        o.n_orbitals = norb;
        o.status = S.status;
    }
}

// getAtomicConfiguration (ElectronicConfiguration.cpp:16-146) as (n,l,alpha,beta) rows
void configuration(int Z, std::vector<std::array<int, 4>>& rows) {
    rows.clear();
    auto add = [&](int n, int l, int e) {
        const int cap = 2 * l + 1;
        const int a = std::min(e, cap);
        rows.push_back({n, l, a, e - a});
    };
    add(1, 0, std::min(Z, 2));
    if (Z >= 3) add(2, 0, std::min(Z - 2, 2));
    if (Z >= 5) add(2, 1, std::min(Z - 4, 6));
    if (Z >= 11) add(3, 0, std::min(Z - 10, 2));
    if (Z >= 13) add(3, 1, std::min(Z - 12, 6));
    if (Z >= 19) {
        int s = Z >= 20 ? 2 : 1;
        if (Z == 24 || Z == 29) s = 1;
        add(4, 0, s);
    }
    if (Z >= 21) {
        int d = Z - 20;
        if (Z == 24) d = 5;
        else if (Z >= 29) d = 10;
        add(3, 2, d);
    }
}

}  // namespace

namespace {

// Builds the run specs, launches the batch and leaves every run's arrays in the WS_RADIAL
// workspace (returned; per_run doubles per run, layout A_* then MAXORB x O_*).
double* run_batch(dft_context* ctx, int nruns, const int* Z, const int* kinds, long points, double rmax,
                  dft_atom_result* results, std::vector<RunSpec>& specs, long long& per_run) {
    if (points < 2) fail(DFT_INVALID_ARGUMENT, "La malla radial debe contener al menos dos puntos.");
    if (points > 12000) fail(DFT_INVALID_ARGUMENT, "at most 12000 radial points per run");
    if (!(rmax > 0.0)) fail(DFT_INVALID_ARGUMENT, "RMAX debe ser mayor que cero.");
    specs.assign(nruns, RunSpec{});
    for (int rr = 0; rr < nruns; ++rr) {
        if (Z[rr] < 1 || Z[rr] > 30) fail(DFT_INVALID_ARGUMENT, "Configuracion atomica no disponible para Z = %d", Z[rr]);
        if (kinds[rr] != 0 && kinds[rr] != 1) fail(DFT_INVALID_ARGUMENT, "unknown functional kind %d", kinds[rr]);
        std::vector<std::array<int, 4>> rows;
        configuration(Z[rr], rows);
        RunSpec& s = specs[rr];
        std::memset(&s, 0, sizeof s);
        s.Z = Z[rr];
        s.kind = kinds[rr];
        s.pivot_eps = ctx->radial_pivot_exp == -14 ? EPS : std::pow(10.0, (double)ctx->radial_pivot_exp);
        int q = 0;
        for (int spin = 0; spin < 2; ++spin) {
            int count_l[4] = {0, 0, 0, 0};
            for (auto& row : rows) {
                const int e = row[2 + spin];
                if (e <= 0) continue;
                s.n[q] = row[0];
                s.l[q] = row[1];
                s.spin[q] = spin;
                s.el[q] = e;
                s.idx[q] = count_l[row[1]]++;
                ++q;
            }
        }
        s.norb = q;
    }
    per_run = (long long)(A_COUNT + MAXORB * O_COUNT) * points;
    double* ws = (double*)ws_get(ctx, WS_RADIAL, sizeof(double) * (size_t)per_run * nruns);
    const size_t spec_bytes = ((sizeof(RunSpec) * nruns + 255) / 256) * 256;  // keep the results 256-B aligned
    char* dbuf = (char*)ws_get(ctx, WS_TMP2, spec_bytes + sizeof(dft_atom_result) * nruns);
    RunSpec* dspec = (RunSpec*)dbuf;
    dft_atom_result* dres = (dft_atom_result*)(dbuf + spec_bytes);
    DFT_CUDA(cudaMemcpyAsync(dspec, specs.data(), sizeof(RunSpec) * nruns, cudaMemcpyHostToDevice, ctx->stream));
    DFT_CUDA(cudaMemsetAsync(dres, 0, sizeof(dft_atom_result) * nruns, ctx->stream));
    const size_t smem = sizeof(double) * (size_t)points;
    if (smem > 48 * 1024)
        DFT_CUDA(cudaFuncSetAttribute(radial_scf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    radial_scf_kernel<<<nruns, RT, smem, ctx->stream>>>(dspec, (int)points, rmax, ws, per_run, dres);
    DFT_LAUNCH_CHECK();
    count_launch(ctx);
    DFT_CUDA(cudaMemcpyAsync(results, dres, sizeof(dft_atom_result) * nruns, cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
    return ws;
}

}  // namespace

void solve_atoms(dft_context* ctx, int nruns, const int* Z, const int* kinds, long points, double rmax,
                 dft_atom_result* results) {
    std::vector<RunSpec> specs;
    long long per_run = 0;
    run_batch(ctx, nruns, Z, kinds, points, rmax, results, specs, per_run);
}

int atomic_orbital_count(int nnuc, const int* Z) {
    int n = 0;
    std::vector<std::array<int, 4>> rows;
    for (int a = 0; a < nnuc; ++a) {
        if (Z[a] < 1 || Z[a] > 30) continue;
        configuration(Z[a], rows);
        for (auto& row : rows)
            if (row[2] > 0 && row[1] <= 2) n += 2 * row[1] + 1;
    }
    return n;
}

void radial_atom_tables(dft_context* ctx, int nz, const int* Z, int kind, long points, double rmax, double* dens,
                        double* orbs, std::vector<std::vector<std::array<int, 2>>>& shells) {
    // elements not solved before on this context (for this functional and radial grid) are
    // solved in one batch and kept; every element is then copied from the kept tables
    long long rbits;
    std::memcpy(&rbits, &rmax, sizeof(rbits));
    auto key = [&](int z) { return std::array<long long, 4>{z, kind, points, rbits}; };
    std::vector<int> todo;
    for (int rr = 0; rr < nz; ++rr)
        if (!ctx->radial_tables.count(key(Z[rr])) && std::find(todo.begin(), todo.end(), Z[rr]) == todo.end())
            todo.push_back(Z[rr]);
    if (!todo.empty()) {
        const int nt = (int)todo.size();
        std::vector<int> kinds(nt, kind);
        std::vector<dft_atom_result> res(nt);
        std::vector<RunSpec> specs;
        long long per_run = 0;
        const double* ws = run_batch(ctx, nt, todo.data(), kinds.data(), points, rmax, res.data(), specs, per_run);
        for (int rr = 0; rr < nt; ++rr) {
            if (res[rr].status != DFT_OK)
                fail((dft_status_t)res[rr].status, "radial atom Z = %d failed (status %d)", todo[rr], res[rr].status);
            RadialTable t;
            const RunSpec& sp = specs[rr];
            for (int q = 0; q < sp.norb; ++q)
                if (sp.spin[q] == 0) t.shells.push_back({sp.n[q], sp.l[q]});  // every occupied alpha (n, l)
            if ((int)t.shells.size() > RADIAL_MAX_SHELLS)
                fail(DFT_INVALID_ARGUMENT, "atom Z = %d has more than %d shells", todo[rr], RADIAL_MAX_SHELLS);
            DFT_CUDA(cudaMalloc(&t.dens, sizeof(double) * points * (1 + RADIAL_MAX_SHELLS)));
            t.orbs = t.dens + points;
            const double* base = ws + (long long)rr * per_run;
            DFT_CUDA(cudaMemcpyAsync(t.dens, base + (long long)A_OD * points, sizeof(double) * points,
                                     cudaMemcpyDeviceToDevice, ctx->stream));
            int k = 0;
            for (int q = 0; q < sp.norb; ++q) {
                if (sp.spin[q] != 0) continue;
                DFT_CUDA(cudaMemcpyAsync(t.orbs + (long long)k * points,
                                         base + (long long)(A_COUNT + q * O_COUNT + O_U) * points,
                                         sizeof(double) * points, cudaMemcpyDeviceToDevice, ctx->stream));
                ++k;
            }
            ctx->radial_tables[key(todo[rr])] = std::move(t);
        }
    }
    shells.assign(nz, {});
    for (int rr = 0; rr < nz; ++rr) {
        const RadialTable& t = ctx->radial_tables.at(key(Z[rr]));
        DFT_CUDA(cudaMemcpyAsync(dens + (long long)rr * points, t.dens, sizeof(double) * points,
                                 cudaMemcpyDeviceToDevice, ctx->stream));
        if (!t.shells.empty())
            DFT_CUDA(cudaMemcpyAsync(orbs + (long long)rr * RADIAL_MAX_SHELLS * points, t.orbs,
                                     sizeof(double) * points * t.shells.size(), cudaMemcpyDeviceToDevice,
                                     ctx->stream));
        shells[rr] = t.shells;
    }
}

}  // namespace dftb
