/*
 * TEST INFRASTRUCTURE — the CPU oracle (see dft_oracle.h).  Plain C99/C11 restatement
 * of the reference algorithms, one function per reference function, each citing the
 * reference file:line it follows.  Loop orders and the order of floating-point
 * operations follow the reference so that results agree to the last bit where the
 * reference's arithmetic is deterministic (built with -ffp-contract=off).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use it.
 */
#define _POSIX_C_SOURCE 199309L
#include "dft_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ---------------------------------------------------------------- errors -- */
static char g_err[256];
const char* oracle_last_error(void) { return g_err; }
#define FAIL(...)                                        \
    do {                                                 \
        snprintf(g_err, sizeof g_err, __VA_ARGS__);      \
        return 1;                                        \
    } while (0)
#define TRY(x)            \
    do {                  \
        int rc_ = (x);    \
        if (rc_) return rc_; \
    } while (0)

/* DFTConstants.h:7-26 */
static const double PI_ = 3.141592653589793238462643383279502884;
static const double EPS_ = 1.0e-14;
static const double RHO_FLOOR_ = 1.0e-20;
static const double EXCHANGE_COEFFICIENT_ = 0.7385587663820223;

static double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
static double maxd(double a, double b) { return a > b ? a : b; }
static double mind(double a, double b) { return a < b ? a : b; }

/* ---------------------------------------------------------------- grid ---- */
/* CartesianGrid.cpp:5-48 (spacing), :115-159 (coordinates, index) */
typedef struct {
    long nx, ny, nz, N;
    double xmin, xmax, ymin, ymax, zmin, zmax, dx, dy, dz;
} grid3;

static int make_grid(const long* n, const double* b, grid3* g) {
    if (n[0] < 2 || n[1] < 2 || n[2] < 2) FAIL("CartesianGrid requires at least two points per dimension.");
    if (b[1] <= b[0] || b[3] <= b[2] || b[5] <= b[4]) FAIL("CartesianGrid requires valid spatial bounds.");
    g->nx = n[0]; g->ny = n[1]; g->nz = n[2];
    g->N = n[0] * n[1] * n[2];
    g->xmin = b[0]; g->xmax = b[1]; g->ymin = b[2]; g->ymax = b[3]; g->zmin = b[4]; g->zmax = b[5];
    g->dx = (g->xmax - g->xmin) / (double)(g->nx - 1);
    g->dy = (g->ymax - g->ymin) / (double)(g->ny - 1);
    g->dz = (g->zmax - g->zmin) / (double)(g->nz - 1);
    return 0;
}
static inline long IDX(const grid3* g, long i, long j, long k) { return (k * g->ny + j) * g->nx + i; }
static inline double GX(const grid3* g, long i) { return g->xmin + (double)i * g->dx; }
static inline double GY(const grid3* g, long j) { return g->ymin + (double)j * g->dy; }
static inline double GZ(const grid3* g, long k) { return g->zmin + (double)k * g->dz; }
static inline double DV(const grid3* g) { return g->dx * g->dy * g->dz; }

/* ============================================================ PZ81 ========= */
/* PZ81.cpp:11-39 parameter sets {A,B,C,D,gamma,beta1,beta2} */
typedef struct { double A, B, C, D, gamma, beta1, beta2; } pz_par;
static const pz_par PZ_U = {0.0311, -0.0480, 0.0020, -0.0116, -0.1423, 1.0529, 0.3334};
static const pz_par PZ_P = {0.01555, -0.0269, 0.0007, -0.0048, -0.0843, 1.3981, 0.2611};

static double pz_rs(double n) { return cbrt(3.0 / (4.0 * PI_ * n)); }                 /* PZ81.cpp:41-50 */
static double pz_ec(double rs, const pz_par* p) {                                       /* PZ81.cpp:52-81 */
    if (rs < 1.0) return p->A * log(rs) + p->B + p->C * rs * log(rs) + p->D * rs;
    double s = sqrt(rs);
    return p->gamma / (1.0 + p->beta1 * s + p->beta2 * rs);
}
static double pz_dec(double rs, const pz_par* p) {                                      /* PZ81.cpp:83-120 */
    if (rs < 1.0) return p->A / rs + p->C * (log(rs) + 1.0) + p->D;
    double s = sqrt(rs);
    double den = 1.0 + p->beta1 * s + p->beta2 * rs;
    double dden = p->beta1 / (2.0 * s) + p->beta2;
    return -p->gamma * dden / (den * den);
}
static double pz_f(double z) {                                                          /* PZ81.cpp:122-149 */
    z = clampd(z, -1.0, 1.0);
    return (pow(1.0 + z, 4.0 / 3.0) + pow(1.0 - z, 4.0 / 3.0) - 2.0) / (pow(2.0, 4.0 / 3.0) - 2.0);
}
static double pz_df(double z) {                                                         /* PZ81.cpp:151-182 */
    z = clampd(z, -1.0, 1.0);
    return 4.0 / 3.0 * (pow(1.0 + z, 1.0 / 3.0) - pow(1.0 - z, 1.0 / 3.0)) / (pow(2.0, 4.0 / 3.0) - 2.0);
}
static double pz_ex(double n) { return -EXCHANGE_COEFFICIENT_ * cbrt(n); }            /* PZ81.cpp:184-190 */
static double pz_sx(double z) {                                                         /* PZ81.cpp:192-213 */
    z = clampd(z, -1.0, 1.0);
    return (pow(1.0 + z, 4.0 / 3.0) + pow(1.0 - z, 4.0 / 3.0)) / 2.0;
}
static double pz_dsx(double z) {                                                        /* PZ81.cpp:215-237 */
    z = clampd(z, -1.0, 1.0);
    return 2.0 / 3.0 * (pow(1.0 + z, 1.0 / 3.0) - pow(1.0 - z, 1.0 / 3.0));
}
static double pz_eps(double n, double z) {                                              /* PZ81.cpp:239-291 */
    double ex = pz_ex(n) * pz_sx(z);
    double rs = pz_rs(n);
    double e0 = pz_ec(rs, &PZ_U), e1 = pz_ec(rs, &PZ_P);
    return ex + (e0 + pz_f(z) * (e1 - e0));
}
static double pz_pot(double n, double a, double bb, int spin) {                        /* PZ81.cpp:293-433 */
    if (n <= RHO_FLOOR_) return 0.0;
    a = maxd(a, 0.0);
    bb = maxd(bb, 0.0);
    double z = clampd((a - bb) / n, -1.0, 1.0);
    double rs = pz_rs(n);
    double ex = pz_ex(n);
    double sx = pz_sx(z), dsx = pz_dsx(z);
    double exs = ex * sx;
    double dexrs = -exs / rs;
    double e0 = pz_ec(rs, &PZ_U), e1 = pz_ec(rs, &PZ_P);
    double d0 = pz_dec(rs, &PZ_U), d1 = pz_dec(rs, &PZ_P);
    double f = pz_f(z), df = pz_df(z);
    double ec = e0 + f * (e1 - e0);
    double decrs = d0 + f * (d1 - d0);
    double exc = exs + ec;
    double dxcrs = dexrs + decrs;
    double dxcz = ex * dsx + df * (e1 - e0);
    double radial = exc - rs * dxcrs / 3.0;
    if (spin == 0) return radial + (1.0 - z) * dxcz;
    return radial - (1.0 + z) * dxcz;
}
static void pz81_evaluate(double na, double nb, double* r) {                          /* PZ81.cpp:437-501 */
    double a = maxd(na, 0.0), bb = maxd(nb, 0.0), n = a + bb;
    r[0] = r[1] = r[2] = r[3] = r[4] = 0.0;
    if (n <= RHO_FLOOR_) return;
    double z = clampd((a - bb) / n, -1.0, 1.0);
    r[0] = pz_eps(n, z);
    r[1] = pz_pot(n, a, bb, 0);
    r[2] = pz_pot(n, a, bb, 1);
}

/* =========================================================== PBE96 ========= */
/* PBE96.cpp:10-54 constants */
static const double THIRD_ = 1.0 / 3.0, FOUR_THIRDS_ = 4.0 / 3.0, TWO_THIRDS_ = 2.0 / 3.0;
static const double KAPPA_ = 0.804, MU_ = 0.2195149727645171;
static const double GAMMA_ = 0.031090690869654895, BETA_ = 0.06672455060314922;
#define DELTA_ (BETA_ / GAMMA_)
static const double SPIN_GAMMA_ = 0.51984209978974632953;
#define SPIN_FZZ_ (8.0 / (9.0 * SPIN_GAMMA_))
static const double ETA_ = 1.0e-12;
static const double EXCHANGE_A_ = -0.73855876638202240588;
static const double KF_COEFFICIENT_ = 3.09366772628014;

static double sgn(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }        /* PBE96.cpp:85-97 */

static double gcor2(double a, double a1, double b1, double b2, double b3, double b4, double srs,
                    double* drs) {                                                      /* PBE96.cpp:99-179 */
    double srs2 = srs * srs;
    double q0 = -2.0 * a * (1.0 + a1 * srs2);
    double q1 = 2.0 * a * srs * (b1 + srs * (b2 + srs * (b3 + b4 * srs)));
    double q2 = log(1.0 + 1.0 / q1);
    double e = q0 * q2;
    double q3 = a * (b1 / srs + 2.0 * b2 + srs * (3.0 * b3 + 4.0 * b4 * srs));
    *drs = -2.0 * a * a1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
    return e;
}

static void pw92(double rs, double z, double* e, double* drs, double* dz) {          /* PBE96.cpp:181-345 */
    double srs = sqrt(rs);
    double eud, epd, ad;
    double eu = gcor2(0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, srs, &eud);
    double ep = gcor2(0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517, srs, &epd);
    double al = gcor2(0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671, srs, &ad);
    double z4 = z * z * z * z;
    double f = (pow(1.0 + z, FOUR_THIRDS_) + pow(1.0 - z, FOUR_THIRDS_) - 2.0) / SPIN_GAMMA_;
    *e = eu * (1.0 - f * z4) + ep * f * z4 - al * f * (1.0 - z4) / SPIN_FZZ_;
    *drs = eud * (1.0 - f * z4) + epd * f * z4 - ad * f * (1.0 - z4) / SPIN_FZZ_;
    double fz = FOUR_THIRDS_ * (pow(1.0 + z, THIRD_) - pow(1.0 - z, THIRD_)) / SPIN_GAMMA_;
    *dz = 4.0 * z * z * z * f * (ep - eu + al / SPIN_FZZ_) + fz * (z4 * ep - z4 * eu - (1.0 - z4) * al / SPIN_FZZ_);
}

/* out: energy density, d/dn, d/d|g|                                                PBE96.cpp:347-444 */
static void pbe_x(double rho, double g, double* out) {
    out[0] = out[1] = out[2] = 0.0;
    if (rho <= 0.0) return;
    double r3 = cbrt(rho);
    double exu = EXCHANGE_A_ * r3;
    double exd = rho * exu;
    double kf = KF_COEFFICIENT_ * r3;
    double den = 2.0 * kf * rho;
    double s = 0.0;
    if (den > 0.0) s = g / den;
    double s2 = s * s;
    double mk = MU_ / KAPPA_;
    double p0 = 1.0 + mk * s2;
    double fx = 1.0 + KAPPA_ - KAPPA_ / p0;
    double fs = 2.0 * KAPPA_ * mk / (p0 * p0);
    out[1] = exu * FOUR_THIRDS_ * (fx - s2 * fs);
    if (g > 0.0) out[2] = EXCHANGE_A_ * 0.161620459673995 * s * fs;
    out[0] = exd * fx;
}

/* out: eps_c, v_a, v_b, d/d|g|                                                     PBE96.cpp:446-810 */
static void pbe_c(double na, double nb, double ga, double gb, double* out) {
    double n = na + nb;
    out[0] = out[1] = out[2] = out[3] = 0.0;
    if (n <= 0.0) return;
    double z = clampd((na - nb) / n, -1.0, 1.0);
    double gm = fabs(ga + gb);
    double kf = cbrt(3.0 * PI_ * PI_ * n);
    double rs = cbrt(3.0 / (4.0 * PI_ * n));
    double phi = 0.5 * (pow(1.0 + z, TWO_THIRDS_) + pow(1.0 - z, TWO_THIRDS_));
    double ks = sqrt(4.0 * kf / PI_);
    double tkp = 2.0 * ks * phi;
    double t = 0.0;
    if (tkp > 0.0) t = gm / (tkp * n);
    double ec, ecrs, ecz;
    pw92(rs, z, &ec, &ecrs, &ecz);
    double phi3 = phi * phi * phi, phi4 = phi3 * phi;
    double ex = -ec / (GAMMA_ * phi3);
    double b;
    if (ex < 700.0) b = DELTA_ / expm1(ex);
    else b = DELTA_ * exp(-ex);
    double b2 = b * b, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
    double q4 = 1.0 + b * t2;
    double q5 = 1.0 + b * t2 + b2 * t4;
    double h = phi3 * (BETA_ / DELTA_) * log(1.0 + DELTA_ * q4 * t2 / q5);
    double rsthrd = rs / 3.0;
    double fac = DELTA_ / b + 1.0;
    double bec = b2 * fac / (BETA_ * phi3);
    double q8 = q5 * q5 + DELTA_ * q4 * q5 * t2;
    double q9 = 1.0 + 2.0 * b * t2;
    double hb = -BETA_ * phi3 * b * t6 * (2.0 + b * t2) / q8;
    double hrs = -rsthrd * hb * bec * ecrs;
    double ht = 2.0 * BETA_ * phi3 * q9 / q8;
    double comm = h + hrs - 7.0 * t2 * ht / 6.0;
    double gz = (pow(1.0 + z + ETA_, -THIRD_) - pow(1.0 - z + ETA_, -THIRD_)) / 3.0;
    double bg = -3.0 * b2 * ec * fac / (BETA_ * phi4);
    double hz = 3.0 * gz * h / phi + hb * (bg * gz + bec * ecz);
    double pref = hz - gz * t2 * ht / phi;
    out[0] = ec + h;
    out[1] = (ec - rs * ecrs / 3.0 - z * ecz) + (ecz) + comm + pref * (1.0 - z);
    out[2] = (ec - rs * ecrs / 3.0 - z * ecz) - (ecz) + comm + pref * (-1.0 - z);
    if (gm > 0.0) out[3] = t * ht / tkp;
}

static void pbe96_evaluate(double na, double nb, double ga, double gb, double* r) {  /* PBE96.cpp:814-966 */
    double a = maxd(na, 0.0), bb = maxd(nb, 0.0), n = a + bb;
    r[0] = r[1] = r[2] = r[3] = r[4] = 0.0;
    if (n <= RHO_FLOOR_) return;
    double xa[3], xb[3], c[4];
    pbe_x(2.0 * a, 2.0 * fabs(ga), xa);
    pbe_x(2.0 * bb, 2.0 * fabs(gb), xb);
    pbe_c(a, bb, ga, gb, c);
    double exd = 0.5 * (xa[0] + xb[0]);
    r[0] = exd / n + c[0];
    r[1] = xa[1] + c[1];
    r[2] = xb[1] + c[2];
    double cs = sgn(ga + gb);
    r[3] = xa[2] * sgn(ga) + c[3] * cs;
    r[4] = xb[2] * sgn(gb) + c[3] * cs;
}

static void xc_eval(int kind, double na, double nb, double ga, double gb, double* r) {
    if (kind == 1) pbe96_evaluate(na, nb, ga, gb, r);
    else pz81_evaluate(na, nb, r);
}

int oracle_xc_evaluate(int kind, long m, const double* na, const double* nb, const double* ga, const double* gb,
                       double* out5) {
    for (long i = 0; i < m; ++i) xc_eval(kind, na[i], nb[i], ga[i], gb[i], out5 + 5 * i);
    return 0;
}

/* ====================================================== 3D operators ======= */
/* applyMolecularKohnShamHamiltonian, KohnShamHamiltonianMolecule.cpp:7-183 */
static void hpsi3(const grid3* g, const double* V, const double* psi, double* out) {
    double ix = 1.0 / (g->dx * g->dx), iy = 1.0 / (g->dy * g->dy), iz = 1.0 / (g->dz * g->dz);
    for (long k = 0; k < g->nz; ++k)
        for (long j = 0; j < g->ny; ++j)
            for (long i = 0; i < g->nx; ++i) {
                long p = IDX(g, i, j, k);
                double c = psi[p];
                double lap = -2.0 * (ix + iy + iz) * c;
                if (i > 0) lap += psi[p - 1] * ix;
                if (i + 1 < g->nx) lap += psi[p + 1] * ix;
                if (j > 0) lap += psi[p - g->nx] * iy;
                if (j + 1 < g->ny) lap += psi[p + g->nx] * iy;
                if (k > 0) lap += psi[p - g->nx * g->ny] * iz;
                if (k + 1 < g->nz) lap += psi[p + g->nx * g->ny] * iz;
                out[p] = -0.5 * lap + V[p] * c;
            }
}

int oracle_apply_hamiltonian(const long* n, const double* b, const double* V, const double* psi, double* out) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    hpsi3(&g, V, psi, out);
    return 0;
}

/* calculateBoundaryPotential, HartreePotentialMolecule.cpp:37-95.  The total charge
 * (:17-35) is recomputed per boundary node by the reference; it is the same sum, so it is
 * computed once here (identical value, same summation order). */
static double boundary_value(const grid3* g, double Q, long i, long j, long k) {
    double x = GX(g, i), y = GY(g, j), z = GZ(g, k);
    double d[6] = {fabs(x - g->xmin), fabs(x - g->xmax), fabs(y - g->ymin),
                   fabs(y - g->ymax), fabs(z - g->zmin), fabs(z - g->zmax)};
    double m2 = INFINITY;
    for (int q = 0; q < 6; ++q) m2 = mind(m2, d[q] * d[q]);
    if (m2 <= 0.0) return 0.0;
    double r = sqrt(x * x + y * y + z * z);
    if (r <= 0.0) return 0.0;
    return Q / r;
}

/* calculateHartreePotential, HartreePotentialMolecule.cpp:99-324: boundary fill, then cold-start
 * Jacobi sweeps with the max|dV| < 1e-8 stop and the silent 10,000-sweep cap (:14-15). */
int oracle_hartree_potential_ex(const long* n, const double* b, const double* rho, double* out, long* sweeps,
                                double* last_diff) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    double ix = 1.0 / (g.dx * g.dx), iy = 1.0 / (g.dy * g.dy), iz = 1.0 / (g.dz * g.dz);
    double den = 2.0 * (ix + iy + iz);
    double* v = calloc((size_t)g.N, sizeof(double));
    double* w;
    double Q = 0.0;
    for (long p = 0; p < g.N; ++p) Q += rho[p];
    Q *= DV(&g);
    for (long k = 0; k < g.nz; ++k)
        for (long j = 0; j < g.ny; ++j)
            for (long i = 0; i < g.nx; ++i)
                if (i == 0 || i + 1 == g.nx || j == 0 || j + 1 == g.ny || k == 0 || k + 1 == g.nz)
                    v[IDX(&g, i, j, k)] = boundary_value(&g, Q, i, j, k);
    w = malloc((size_t)g.N * sizeof(double));
    memcpy(w, v, (size_t)g.N * sizeof(double));
    long it, sx = g.nx, sxy = g.nx * g.ny, done = 0;
    double md = 0.0;
    for (it = 0; it < 10000; ++it) {
        md = 0.0;
        for (long k = 1; k + 1 < g.nz; ++k)
            for (long j = 1; j + 1 < g.ny; ++j)
                for (long i = 1; i + 1 < g.nx; ++i) {
                    long p = IDX(&g, i, j, k);
                    double src = 4.0 * PI_ * rho[p];
                    w[p] = (ix * (v[p - 1] + v[p + 1]) + iy * (v[p - sx] + v[p + sx]) + iz * (v[p - sxy] + v[p + sxy]) +
                            src) / den;
                    md = maxd(md, fabs(w[p] - v[p]));
                }
        double* t = v;
        v = w;
        w = t;
        if (md < 1.0e-8) {
            done = 1;
            break;
        }
    }
    memcpy(out, v, (size_t)g.N * sizeof(double));
    if (sweeps) *sweeps = done ? it + 1 : it;
    if (last_diff) *last_diff = md;
    free(v);
    free(w);
    return 0;
}

int oracle_hartree_potential(const long* n, const double* b, const double* rho, double* out) {
    return oracle_hartree_potential_ex(n, b, rho, out, NULL, NULL);
}

/* calculateHartreeEnergy, HartreePotentialMolecule.cpp:326-379 */
int oracle_hartree_energy(const long* n, const double* b, const double* rho, const double* vh, double* e) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    double s = 0.0;
    for (long p = 0; p < g.N; ++p) s += rho[p] * vh[p];
    *e = 0.5 * s * DV(&g);
    return 0;
}

/* calculateCartesianDerivative, ExchangeCorrelationMolecule.cpp:11-170 */
static double deriv(const grid3* g, const double* f, long i, long j, long k, int dir) {
    if (dir == 0) {
        if (i == 0) return (f[IDX(g, i + 1, j, k)] - f[IDX(g, i, j, k)]) / g->dx;
        if (i == g->nx - 1) return (f[IDX(g, i, j, k)] - f[IDX(g, i - 1, j, k)]) / g->dx;
        return (f[IDX(g, i + 1, j, k)] - f[IDX(g, i - 1, j, k)]) / (2.0 * g->dx);
    }
    if (dir == 1) {
        if (j == 0) return (f[IDX(g, i, j + 1, k)] - f[IDX(g, i, j, k)]) / g->dy;
        if (j == g->ny - 1) return (f[IDX(g, i, j, k)] - f[IDX(g, i, j - 1, k)]) / g->dy;
        return (f[IDX(g, i, j + 1, k)] - f[IDX(g, i, j - 1, k)]) / (2.0 * g->dy);
    }
    if (k == 0) return (f[IDX(g, i, j, k + 1)] - f[IDX(g, i, j, k)]) / g->dz;
    if (k == g->nz - 1) return (f[IDX(g, i, j, k)] - f[IDX(g, i, j, k - 1)]) / g->dz;
    return (f[IDX(g, i, j, k + 1)] - f[IDX(g, i, j, k - 1)]) / (2.0 * g->dz);
}

/* calculateGradientMagnitude, ExchangeCorrelationMolecule.cpp:172-214 */
static double gradmag(const grid3* g, const double* f, long i, long j, long k) {
    double gx = deriv(g, f, i, j, k, 0), gy = deriv(g, f, i, j, k, 1), gz = deriv(g, f, i, j, k, 2);
    return sqrt(gx * gx + gy * gy + gz * gz);
}

/* calculateCartesianDivergence, ExchangeCorrelationMolecule.cpp:216-572 */
static double divergence(const grid3* g, const double* c, const double* f, long i, long j, long k) {
    long p = IDX(g, i, j, k);
    double cc = c[p];
    double fx = cc * deriv(g, f, i, j, k, 0), fy = cc * deriv(g, f, i, j, k, 1), fz = cc * deriv(g, f, i, j, k, 2);
    double dxv, dyv, dzv;
    if (i == 0) dxv = (c[IDX(g, i + 1, j, k)] * deriv(g, f, i + 1, j, k, 0) - fx) / g->dx;
    else if (i == g->nx - 1) dxv = (fx - c[IDX(g, i - 1, j, k)] * deriv(g, f, i - 1, j, k, 0)) / g->dx;
    else
        dxv = (c[IDX(g, i + 1, j, k)] * deriv(g, f, i + 1, j, k, 0) - c[IDX(g, i - 1, j, k)] * deriv(g, f, i - 1, j, k, 0)) /
              (2.0 * g->dx);
    if (j == 0) dyv = (c[IDX(g, i, j + 1, k)] * deriv(g, f, i, j + 1, k, 1) - fy) / g->dy;
    else if (j == g->ny - 1) dyv = (fy - c[IDX(g, i, j - 1, k)] * deriv(g, f, i, j - 1, k, 1)) / g->dy;
    else
        dyv = (c[IDX(g, i, j + 1, k)] * deriv(g, f, i, j + 1, k, 1) - c[IDX(g, i, j - 1, k)] * deriv(g, f, i, j - 1, k, 1)) /
              (2.0 * g->dy);
    if (k == 0) dzv = (c[IDX(g, i, j, k + 1)] * deriv(g, f, i, j, k + 1, 2) - fz) / g->dz;
    else if (k == g->nz - 1) dzv = (fz - c[IDX(g, i, j, k - 1)] * deriv(g, f, i, j, k - 1, 2)) / g->dz;
    else
        dzv = (c[IDX(g, i, j, k + 1)] * deriv(g, f, i, j, k + 1, 2) - c[IDX(g, i, j, k - 1)] * deriv(g, f, i, j, k - 1, 2)) /
              (2.0 * g->dz);
    return dxv + dyv + dzv;
}

/* calculateMolecularSpinExchangeCorrelationPotential, ExchangeCorrelationMolecule.cpp:576-747 */
static int xc_potential3(int kind, const grid3* g, const double* na, const double* nb, int spin, double* out) {
    if (spin != 0 && spin != 1) FAIL("El canal de spin debe ser 0 (alpha) o 1 (beta).");
    double* dd = calloc((size_t)g->N, sizeof(double));
    double* cc = calloc((size_t)g->N, sizeof(double));
    for (long k = 0; k < g->nz; ++k)
        for (long j = 0; j < g->ny; ++j)
            for (long i = 0; i < g->nx; ++i) {
                long p = IDX(g, i, j, k);
                if (na[p] + nb[p] <= RHO_FLOOR_) continue;
                double r[5];
                xc_eval(kind, na[p], nb[p], gradmag(g, na, i, j, k), gradmag(g, nb, i, j, k), r);
                dd[p] = spin == 0 ? r[1] : r[2];
                cc[p] = spin == 0 ? r[3] : r[4];
            }
    const double* f = spin == 0 ? na : nb;
    for (long k = 0; k < g->nz; ++k)
        for (long j = 0; j < g->ny; ++j)
            for (long i = 0; i < g->nx; ++i) {
                long p = IDX(g, i, j, k);
                if (na[p] + nb[p] <= RHO_FLOOR_) {
                    out[p] = 0.0;
                    continue;
                }
                out[p] = dd[p] - divergence(g, cc, f, i, j, k);
            }
    free(dd);
    free(cc);
    return 0;
}

int oracle_xc_potential(int kind, const long* n, const double* b, const double* na, const double* nb, int spin,
                        double* out) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    return xc_potential3(kind, &g, na, nb, spin, out);
}

/* calculateMolecularExchangeCorrelationEnergy, ExchangeCorrelationMolecule.cpp:749-842 */
static double xc_energy3(int kind, const grid3* g, const double* na, const double* nb) {
    double dv = DV(g), e = 0.0;
    for (long k = 0; k < g->nz; ++k)
        for (long j = 0; j < g->ny; ++j)
            for (long i = 0; i < g->nx; ++i) {
                long p = IDX(g, i, j, k);
                double n = na[p] + nb[p];
                if (n <= RHO_FLOOR_) continue;
                double r[5];
                xc_eval(kind, na[p], nb[p], gradmag(g, na, i, j, k), gradmag(g, nb, i, j, k), r);
                e += n * r[0] * dv;
            }
    return e;
}

int oracle_xc_energy(int kind, const long* n, const double* b, const double* na, const double* nb, double* e) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    *e = xc_energy3(kind, &g, na, nb);
    return 0;
}

/* NuclearPotential::calculate / calculateAtPoint, NuclearPotential.cpp:6-76 */
int oracle_nuclear_potential(const long* n, const double* b, int nnuc, const int* Z, const double* xyz,
                             double* out) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    for (long k = 0; k < g.nz; ++k) {
        double z = GZ(&g, k);
        for (long j = 0; j < g.ny; ++j) {
            double y = GY(&g, j);
            for (long i = 0; i < g.nx; ++i) {
                double x = GX(&g, i), v = 0.0;
                for (int a = 0; a < nnuc; ++a) {
                    double dx = x - xyz[3 * a], dy = y - xyz[3 * a + 1], dz = z - xyz[3 * a + 2];
                    double d2 = dx * dx + dy * dy + dz * dz;
                    if (d2 == 0.0) FAIL("NuclearPotential is singular at a nuclear position.");
                    v -= (double)Z[a] / sqrt(d2);
                }
                out[IDX(&g, i, j, k)] = v;
            }
        }
    }
    return 0;
}

/* NuclearRepulsion::calculate, NuclearRepulsion.cpp:6-54 */
int oracle_nuclear_repulsion(int nnuc, const int* Z, const double* xyz, double* e) {
    double s = 0.0;
    for (int a = 0; a < nnuc; ++a)
        for (int c = a + 1; c < nnuc; ++c) {
            double dx = xyz[3 * a] - xyz[3 * c], dy = xyz[3 * a + 1] - xyz[3 * c + 1], dz = xyz[3 * a + 2] - xyz[3 * c + 2];
            double d2 = dx * dx + dy * dy + dz * dz;
            if (d2 == 0.0) FAIL("NuclearRepulsion is undefined for coincident nuclei.");
            s += (double)Z[a] * (double)Z[c] / sqrt(d2);
        }
    *e = s;
    return 0;
}

/* calculateMolecularKineticEnergy, TotalEnergyMolecule.cpp:13-199 (face stencil of existing neighbours) */
static double kinetic3(const grid3* g, int nbands, const double* psi, const int* el) {
    double dv = DV(g), e = 0.0;
    double hx = g->dx * g->dx, hy = g->dy * g->dy, hz = g->dz * g->dz;
    for (int bnd = 0; bnd < nbands; ++bnd) {
        if (el[bnd] <= 0) continue;
        const double* f = psi + (size_t)bnd * g->N;
        double oe = 0.0;
        for (long k = 0; k < g->nz; ++k)
            for (long j = 0; j < g->ny; ++j)
                for (long i = 0; i < g->nx; ++i) {
                    long p = IDX(g, i, j, k);
                    double c = f[p], lap = 0.0;
                    if (i > 0) lap += (f[p - 1] - c) / hx;
                    if (i + 1 < g->nx) lap += (f[p + 1] - c) / hx;
                    if (j > 0) lap += (f[p - g->nx] - c) / hy;
                    if (j + 1 < g->ny) lap += (f[p + g->nx] - c) / hy;
                    if (k > 0) lap += (f[p - g->nx * g->ny] - c) / hz;
                    if (k + 1 < g->nz) lap += (f[p + g->nx * g->ny] - c) / hz;
                    oe += c * (-0.5 * lap) * dv;
                }
        e += (double)el[bnd] * oe;
    }
    return e;
}

int oracle_kinetic_energy(const long* n, const double* b, int nbands, const double* psi, const int* electrons,
                          double* e) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    *e = kinetic3(&g, nbands, psi, electrons);
    return 0;
}

/* calculateMolecularSpinDensity, ElectronDensityMolecule.cpp:5-76 */
int oracle_spin_density(long N, int nbands, const double* psi, const int* electrons, double* out) {
    if (nbands <= 0) FAIL("La lista de orbitales moleculares no puede estar vacia.");
    for (long p = 0; p < N; ++p) out[p] = 0.0;
    for (int bnd = 0; bnd < nbands; ++bnd) {
        if (electrons[bnd] <= 0) continue;
        const double* f = psi + (size_t)bnd * N;
        for (long p = 0; p < N; ++p) out[p] += (double)electrons[bnd] * f[p] * f[p];
    }
    return 0;
}

/* calculateMolecularDensityDifference, MolecularSCFHelpers.cpp:46-95 */
static double ddiff3(const grid3* g, const double* o, const double* nw) {
    double dv = DV(g), d2 = 0.0, n2 = 0.0;
    for (long p = 0; p < g->N; ++p) {
        double d = nw[p] - o[p];
        d2 += d * d;
        n2 += nw[p] * nw[p];
    }
    double dn = sqrt(d2 * dv), nn = sqrt(n2 * dv);
    if (nn <= EPS_) return dn;
    return dn / nn;
}

int oracle_density_difference(const long* n, const double* b, const double* old_d, const double* new_d,
                              double* out) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    *out = ddiff3(&g, old_d, new_d);
    return 0;
}

/* calculateMaximumMolecularKSResidual, MolecularSCFHelpers.cpp:119-183 (one potential for all bands) */
static double ksres3(const grid3* g, const double* V, int nbands, const double* psi, const double* eig, double* tmp) {
    double dv = DV(g), m = 0.0;
    for (int bnd = 0; bnd < nbands; ++bnd) {
        const double* f = psi + (size_t)bnd * g->N;
        hpsi3(g, V, f, tmp);
        double s = 0.0;
        for (long p = 0; p < g->N; ++p) {
            double r = tmp[p] - eig[bnd] * f[p];
            s += r * r;
        }
        m = maxd(m, sqrt(s * dv));
    }
    return m;
}

int oracle_ks_residual(const long* n, const double* b, const double* V, int nbands, const double* psi,
                       const double* eig, double* out) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    double* tmp = malloc((size_t)g.N * sizeof(double));
    *out = ksres3(&g, V, nbands, psi, eig, tmp);
    free(tmp);
    return 0;
}

/* ================================================ state-by-state Davidson === */
/* EigenvalueSolverMolecule.cpp:19-25 */
#define MO_TOL 1.0e-7
#define SUB_TOL 1.0e-12
#define VEC_TOL2 1.0e-20
#define MAXSUB 16
#define JAC_TOL 1.0e-13
#define JAC_MAXIT 10000
#define DEN_TOL 1.0e-10

static double vdot(long N, const double* a, const double* b) {                       /* NumericalMethods.cpp:9-26 */
    double s = 0.0;
    for (long i = 0; i < N; ++i) s += a[i] * b[i];
    return s;
}
static double wdot(long N, const double* a, const double* b, double dv) { return dv * vdot(N, a, b); } /* :35-47 */
static int valid_norm(long N, const double* v, double dv, double tol2) {                               /* :56-65 */
    double n2 = wdot(N, v, v, dv);
    return isfinite(n2) && n2 > tol2;
}
static int vnormalize(long N, double* v, double dv, double tol2) {                                     /* :67-87 */
    double n2 = wdot(N, v, v, dv);
    if (!isfinite(n2) || n2 <= tol2) FAIL("No se puede normalizar el vector molecular.");
    double nn = sqrt(n2);
    for (long i = 0; i < N; ++i) v[i] /= nn;
    return 0;
}
static void orth_basis(long N, double* v, double** basis, int nb, double dv) {                       /* :89-103 */
    for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < nb; ++q) {
            double pr = wdot(N, basis[q], v, dv);
            for (long i = 0; i < N; ++i) v[i] -= pr * basis[q][i];
        }
}
static int orth_orbitals(long N, double* v, const double* orbs, int no, double dv) {                 /* :105-131 */
    for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < no; ++q) {
            const double* o = orbs + (size_t)q * N;
            double on = wdot(N, o, o, dv);
            if (!isfinite(on) || on <= VEC_TOL2) FAIL("Un orbital molecular previo no es valido.");
            double pr = wdot(N, o, v, dv) / on;
            for (long i = 0; i < N; ++i) v[i] -= pr * o[i];
        }
    return 0;
}

/* buildInitialVector, EigenvalueSolverMolecule.cpp:177-283 */
static void initial_vector(const grid3* g, long idx, double* v) {
    double cx = 0.5 * (g->xmin + g->xmax), cy = 0.5 * (g->ymin + g->ymax), cz = 0.5 * (g->zmin + g->zmax);
    double sigma = 0.8 + 0.18 * (double)idx;
    double fac = 1.0 / (2.0 * sigma * sigma);
    long mode = idx % 9;
    for (long k = 0; k < g->nz; ++k) {
        double z = GZ(g, k) - cz;
        for (long j = 0; j < g->ny; ++j) {
            double y = GY(g, j) - cy;
            for (long i = 0; i < g->nx; ++i) {
                double x = GX(g, i) - cx;
                double r2 = x * x + y * y + z * z;
                double ga = exp(-r2 * fac), pl = 1.0;
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
                v[k * g->nx * g->ny + j * g->nx + i] = pl * ga;
            }
        }
    }
}

/* diagonalize, EigenvalueSolverMolecule.cpp:290-449: cyclic-by-largest Jacobi, lowest pair.
 * a is n x n row-major and is destroyed. */
static int jacobi_lowest(int n, double* a, double* theta, double* vec) {
    double V[MAXSUB * MAXSUB];
    for (int i = 0; i < n * n; ++i) V[i] = 0.0;
    for (int i = 0; i < n; ++i) V[i * n + i] = 1.0;
    for (int it = 0; it < JAC_MAXIT; ++it) {
        double mx = 0.0;
        int p = 0, q = 0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) {
                double v = fabs(a[i * n + j]);
                if (v > mx) {
                    mx = v;
                    p = i;
                    q = j;
                }
            }
        if (mx <= JAC_TOL) break;
        double app = a[p * n + p], aqq = a[q * n + q], apq = a[p * n + q];
        if (apq == 0.0) continue;
        double tau = (aqq - app) / (2.0 * apq);
        double t = copysign(1.0 / (fabs(tau) + sqrt(1.0 + tau * tau)), tau);
        double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        a[p * n + p] = app - t * apq;
        a[q * n + q] = aqq + t * apq;
        a[p * n + q] = 0.0;
        a[q * n + p] = 0.0;
        for (int k = 0; k < n; ++k) {
            if (k == p || k == q) continue;
            double mkp = a[k * n + p], mkq = a[k * n + q];
            a[k * n + p] = c * mkp - s * mkq;
            a[p * n + k] = a[k * n + p];
            a[k * n + q] = s * mkp + c * mkq;
            a[q * n + k] = a[k * n + q];
        }
        for (int k = 0; k < n; ++k) {
            double vkp = V[k * n + p], vkq = V[k * n + q];
            V[k * n + p] = c * vkp - s * vkq;
            V[k * n + q] = s * vkp + c * vkq;
        }
    }
    int idx = 0;
    for (int i = 1; i < n; ++i)
        if (a[i * n + i] < a[idx * n + idx]) idx = i;
    double nn = 0.0;
    for (int i = 0; i < n; ++i) {
        vec[i] = V[i * n + idx];
        nn += vec[i] * vec[i];
    }
    nn = sqrt(nn);
    if (!isfinite(nn) || nn <= EPS_) FAIL("Autovector denso invalido.");
    for (int i = 0; i < n; ++i) vec[i] /= nn;
    *theta = a[idx * n + idx];
    return 0;
}

/* buildIndependentVector, EigenvalueSolverMolecule.cpp:557-590 */
static int independent_vector(const grid3* g, long idx, const double* orbs, int no, double dv, double* out,
                              int* ok) {
    *ok = 0;
    for (long seed = idx; seed < idx + 64; ++seed) {
        initial_vector(g, seed, out);
        TRY(orth_orbitals(g->N, out, orbs, no, dv));
        if (!valid_norm(g->N, out, dv, VEC_TOL2)) continue;
        TRY(vnormalize(g->N, out, dv, VEC_TOL2));
        *ok = 1;
        return 0;
    }
    return 0;
}

/* appendIndependentCorrection, EigenvalueSolverMolecule.cpp:626-662 */
static int append_correction(long N, double* c, const double* orbs, int no, double** basis, int nb, double dv,
                             int* ok) {
    TRY(orth_orbitals(N, c, orbs, no, dv));
    orth_basis(N, c, basis, nb, dv);
    *ok = 0;
    if (!valid_norm(N, c, dv, SUB_TOL * SUB_TOL)) return 0;
    TRY(vnormalize(N, c, dv, SUB_TOL * SUB_TOL));
    *ok = 1;
    return 0;
}

typedef struct {
    double* basis[MAXSUB];
    double* hbasis[MAXSUB];
    double* ritz;
    double* hritz;
    double* res;
    double* corr;
    double* diag;
    double* tmp;
} dav_ws;

/* solveMolecularOrbital, EigenvalueSolverMolecule.cpp:666-1231: single-vector Davidson for orbital
 * `idx`, deflated against the `no` previous orbitals; writes psi_out and eig. */
static int solve_orbital3(const grid3* g, const double* V, long idx, const double* orbs, int no,
                          const double* guess, double* psi_out, double* eig, dav_ws* w) {
    const long N = g->N;
    const double dv = DV(g);
    double kin = 1.0 / (g->dx * g->dx) + 1.0 / (g->dy * g->dy) + 1.0 / (g->dz * g->dz);
    for (long p = 0; p < N; ++p) w->diag[p] = kin + V[p];                          /* :483-519 */
    int nb = 0, nh = 0, ok = 0;
    double P[MAXSUB * MAXSUB];
    double A[MAXSUB * MAXSUB];
    double y[MAXSUB];
    /* buildInitialFromPrevious :592-624, else buildIndependentVector */
    int have = 0;
    if (guess) {
        int fin = 1;
        memcpy(w->basis[0], guess, (size_t)N * sizeof(double));
        for (long p = 0; p < N; ++p)
            if (!isfinite(w->basis[0][p])) fin = 0;
        if (fin) {
            TRY(orth_orbitals(N, w->basis[0], orbs, no, dv));
            if (valid_norm(N, w->basis[0], dv, VEC_TOL2)) {
                TRY(vnormalize(N, w->basis[0], dv, VEC_TOL2));
                have = 1;
            }
        }
    }
    if (!have) {
        TRY(independent_vector(g, idx, orbs, no, dv, w->basis[0], &ok));
        if (!ok) FAIL("No se pudo construir el vector inicial.");
    }
    nb = 1;
    long happ = 0;
    double fe = INFINITY, fr = INFINITY;
    int have_final = 0;
    while (happ < 5000) {
        if (nh < nb) {
            int ix = nh;
            hpsi3(g, V, w->basis[ix], w->hbasis[ix]);
            ++nh;
            ++happ;
            /* the projected matrix keeps earlier entries; new entries are zero until set */
            for (int i = 0; i <= ix; ++i) {
                double v = wdot(N, w->basis[i], w->hbasis[ix], dv);
                P[i * MAXSUB + ix] = v;
                P[ix * MAXSUB + i] = v;
            }
        }
        int n = nb;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) A[i * n + j] = P[i * MAXSUB + j];
        double th;
        TRY(jacobi_lowest(n, A, &th, y));
        /* combine :451-481 */
        for (long p = 0; p < N; ++p) w->ritz[p] = 0.0;
        for (int q = 0; q < n; ++q)
            for (long p = 0; p < N; ++p) w->ritz[p] += y[q] * w->basis[q][p];
        if (!valid_norm(N, w->ritz, dv, VEC_TOL2)) FAIL("El vector de Ritz es numericamente nulo.");
        TRY(vnormalize(N, w->ritz, dv, VEC_TOL2));
        hpsi3(g, V, w->ritz, w->hritz);
        ++happ;
        /* rayleigh :133-149, residualNorm :151-175 */
        double den = wdot(N, w->ritz, w->ritz, dv);
        if (!isfinite(den) || den <= VEC_TOL2) FAIL("Norma invalida en el cociente de Rayleigh.");
        fe = wdot(N, w->ritz, w->hritz, dv) / den;
        for (long p = 0; p < N; ++p) w->res[p] = w->hritz[p] - fe * w->ritz[p];
        double r2 = wdot(N, w->res, w->res, dv);
        fr = isfinite(r2) ? sqrt(r2) : INFINITY;
        memcpy(psi_out, w->ritz, (size_t)N * sizeof(double));
        have_final = 1;
        if (fr < MO_TOL) break;
        for (long p = 0; p < N; ++p) w->res[p] = w->hritz[p] - fe * w->ritz[p];
        TRY(orth_orbitals(N, w->res, orbs, no, dv));
        double* add = w->corr;
        if (!valid_norm(N, w->res, dv, SUB_TOL * SUB_TOL)) {
            TRY(independent_vector(g, idx + nb, orbs, no, dv, add, &ok));
            if (!ok) FAIL("No se pudo construir una nueva direccion independiente para Davidson.");
            orth_basis(N, add, w->basis, nb, dv);
            if (!valid_norm(N, add, dv, SUB_TOL * SUB_TOL)) FAIL("La nueva direccion Davidson es numericamente dependiente.");
            TRY(vnormalize(N, add, dv, SUB_TOL * SUB_TOL));
            if (nb < MAXSUB) {
                memcpy(w->basis[nb], add, (size_t)N * sizeof(double));
                ++nb;
                continue;
            }
        } else {
            /* davidsonCorrection :521-555 */
            for (long p = 0; p < N; ++p) {
                double d = fe - w->diag[p];
                add[p] = (!isfinite(d) || fabs(d) < DEN_TOL) ? w->res[p] : w->res[p] / d;
            }
            TRY(append_correction(N, add, orbs, no, w->basis, nb, dv, &ok));
            if (!ok) {
                memcpy(add, w->res, (size_t)N * sizeof(double));
                TRY(append_correction(N, add, orbs, no, w->basis, nb, dv, &ok));
                if (!ok) {
                    TRY(independent_vector(g, idx + nb, orbs, no, dv, add, &ok));
                    if (!ok) FAIL("No se pudo construir una direccion de expansion Davidson valida.");
                    orth_basis(N, add, w->basis, nb, dv);
                    if (!valid_norm(N, add, dv, SUB_TOL * SUB_TOL))
                        FAIL("La direccion de expansion Davidson es numericamente dependiente.");
                    TRY(vnormalize(N, add, dv, SUB_TOL * SUB_TOL));
                }
            }
            if (nb < MAXSUB) {
                memcpy(w->basis[nb], add, (size_t)N * sizeof(double));
                ++nb;
                continue;
            }
        }
        /* thick restart to {ritz, new direction} (:1107-1190 and :972-1016) */
        if (happ >= 5000) break;
        hpsi3(g, V, add, w->tmp);
        ++happ;
        memcpy(w->basis[0], w->ritz, (size_t)N * sizeof(double));
        memcpy(w->basis[1], add, (size_t)N * sizeof(double));
        memcpy(w->hbasis[0], w->hritz, (size_t)N * sizeof(double));
        memcpy(w->hbasis[1], w->tmp, (size_t)N * sizeof(double));
        nb = nh = 2;
        P[0] = wdot(N, w->basis[0], w->hbasis[0], dv);
        P[1] = wdot(N, w->basis[0], w->hbasis[1], dv);
        P[MAXSUB] = P[1];
        P[MAXSUB + 1] = wdot(N, w->basis[1], w->hbasis[1], dv);
    }
    if (!have_final || fr >= MO_TOL)
        FAIL("El orbital molecular no convergio. Orbital = %ld, residual = %f", idx, fr);
    *eig = fe;
    return 0;
}

static dav_ws* dav_alloc(long N) {
    dav_ws* w = calloc(1, sizeof(dav_ws));
    for (int i = 0; i < MAXSUB; ++i) {
        w->basis[i] = malloc((size_t)N * sizeof(double));
        w->hbasis[i] = malloc((size_t)N * sizeof(double));
    }
    w->ritz = malloc((size_t)N * sizeof(double));
    w->hritz = malloc((size_t)N * sizeof(double));
    w->res = malloc((size_t)N * sizeof(double));
    w->corr = malloc((size_t)N * sizeof(double));
    w->diag = malloc((size_t)N * sizeof(double));
    w->tmp = malloc((size_t)N * sizeof(double));
    return w;
}
static void dav_free(dav_ws* w) {
    for (int i = 0; i < MAXSUB; ++i) {
        free(w->basis[i]);
        free(w->hbasis[i]);
    }
    free(w->ritz); free(w->hritz); free(w->res); free(w->corr); free(w->diag); free(w->tmp);
    free(w);
}

/* solveMolecularOrbitals, EigenvalueSolverMolecule.cpp:1233-1300 */
static int solve_orbitals3(const grid3* g, const double* V, int norb, const double* init, double* psi, double* eig) {
    if (norb <= 0) FAIL("El numero de orbitales debe ser mayor que cero.");
    dav_ws* w = dav_alloc(g->N);
    int rc = 0;
    for (int i = 0; i < norb && !rc; ++i)
        rc = solve_orbital3(g, V, i, psi, i, init ? init + (size_t)i * g->N : NULL, psi + (size_t)i * g->N, eig + i, w);
    dav_free(w);
    return rc;
}

int oracle_solve_orbitals(const long* n, const double* b, const double* V, int norb, const double* init,
                          double* psi_out, double* eig_out) {
    grid3 g;
    TRY(make_grid(n, b, &g));
    return solve_orbitals3(&g, V, norb, init, psi_out, eig_out);
}

/* ====================================================== molecular SCF ===== */
/* solveMolecularSelfConsistentField, SelfConsistentFieldMolecule.cpp:50-561, with
 * executeMolecularSCFIteration (MolecularSCFIteration.cpp:12-252) inlined.  Mixing constants
 * SelfConsistentFieldMolecule.cpp:27-31; tolerances DFTConstants.h:15-19. */
static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int scf_run(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int charge,
                   int multiplicity, int kind, double* energies6, double* stats4, int n_eig, double* eig_out,
                   double* dens_out, int max_it, double* seconds2) {
    const double t_begin = now_s();
    double t_init = 0.0;
    grid3 g;
    TRY(make_grid(n, b, &g));
    if (nnuc <= 0) FAIL("La molecula debe contener al menos un nucleo.");
    if (multiplicity < 1) FAIL("La multiplicidad electronica debe ser al menos 1.");
    int nuc = 0;
    for (int a = 0; a < nnuc; ++a) nuc += Z[a];
    int ne = nuc - charge;
    if (ne < 0) FAIL("La carga molecular produce un numero negativo de electrones.");
    if (ne == 0) FAIL("El SCF molecular requiere al menos un electron.");
    int sd = multiplicity - 1;
    if (sd > ne) FAIL("La multiplicidad electronica es incompatible con el numero de electrones.");
    if ((ne - sd) % 2 != 0) FAIL("La multiplicidad electronica es incompatible con la paridad del numero de electrones.");
    int na_ = (ne + sd) / 2, nb_ = (ne - sd) / 2;
    int closed = multiplicity == 1;
    if (nb_ == 0) FAIL("El numero de orbitales debe ser mayor que cero.");
    const long N = g.N;
    const double dv = DV(&g);
    size_t B = (size_t)N * sizeof(double);
    double *vext = malloc(B), *da = malloc(B), *db = malloc(B), *rho = malloc(B), *vh = malloc(B);
    double *vxa = malloc(B), *vxb = malloc(B), *va = malloc(B), *vb = malloc(B);
    double *oa = malloc(B), *ob = malloc(B), *orho = malloc(B), *ovh = malloc(B), *tmp = malloc(B);
    /* alpha then beta orbitals in one block: the energy sums replay the reference's orbital order */
    double *pall = malloc(B * (na_ + nb_)), *prev_a = malloc(B * na_), *prev_b = malloc(B * nb_);
    double *pa = pall, *pb = pall + (size_t)na_ * N;
    double *ea = malloc(sizeof(double) * na_), *eb = malloc(sizeof(double) * nb_);
    int* ones = malloc(sizeof(int) * (na_ + nb_));
    for (int i = 0; i < na_ + nb_; ++i) ones[i] = 1;
    int rc = oracle_nuclear_potential(n, b, nnuc, Z, xyz, vext);
    double enn = 0.0;
    if (!rc) rc = oracle_nuclear_repulsion(nnuc, Z, xyz, &enn);
    /* buildInitialMolecularDensities, MolecularSCFHelpers.cpp:515-579 */
    if (!rc) rc = solve_orbitals3(&g, vext, na_, NULL, prev_a, ea);
    if (!rc) {
        if (closed) memcpy(prev_b, prev_a, B * nb_);
        else rc = solve_orbitals3(&g, vext, nb_, NULL, prev_b, eb);
    }
    if (!rc) {
        oracle_spin_density(N, na_, prev_a, ones, da);
        oracle_spin_density(N, nb_, prev_b, ones, db);
    }
    double prevE = INFINITY, prevD = INFINITY, mixing = 0.25;
    int it = 0, conv = 0;
    double E[6] = {0}, effd = 0, resid = 0;
    t_init = now_s();
    for (it = 1; !rc && it <= max_it; ++it) {
        double imix = mixing;
        for (long p = 0; p < N; ++p) rho[p] = da[p] + db[p];
        if ((rc = oracle_hartree_potential(n, b, rho, vh))) break;
        if ((rc = xc_potential3(kind, &g, da, db, 0, vxa))) break;
        if (closed) memcpy(vxb, vxa, B);
        else if ((rc = xc_potential3(kind, &g, da, db, 1, vxb))) break;
        for (long p = 0; p < N; ++p) {
            va[p] = vext[p] + vh[p] + vxa[p];
            vb[p] = vext[p] + vh[p] + vxb[p];
        }
        if ((rc = solve_orbitals3(&g, va, na_, prev_a, pa, ea))) break;
        if (closed) {
            memcpy(pb, pa, B * nb_);
            memcpy(eb, ea, sizeof(double) * nb_);
        } else if ((rc = solve_orbitals3(&g, vb, nb_, prev_b, pb, eb))) break;
        oracle_spin_density(N, na_, pa, ones, oa);
        oracle_spin_density(N, nb_, pb, ones, ob);
        for (long p = 0; p < N; ++p) orho[p] = oa[p] + ob[p];
        if ((rc = oracle_hartree_potential(n, b, orho, ovh))) break;
        /* calculateMolecularTotalEnergy, TotalEnergyMolecule.cpp:237-333 (alpha then beta orbitals) */
        double T = kinetic3(&g, na_ + nb_, pall, ones);
        double eext = 0.0;
        for (long p = 0; p < N; ++p) eext += orho[p] * vext[p] * dv;
        double eh;
        oracle_hartree_energy(n, b, orho, ovh, &eh);
        double exc = xc_energy3(kind, &g, oa, ob);
        E[0] = T; E[1] = eext; E[2] = eh; E[3] = exc; E[4] = enn;
        E[5] = T + eext + eh + exc + enn;
        double dd = ddiff3(&g, rho, orho);
        double sdd = maxd(ddiff3(&g, da, oa), ddiff3(&g, db, ob));
        effd = maxd(dd, sdd);
        resid = maxd(ksres3(&g, va, na_, pa, ea, tmp), ksres3(&g, vb, nb_, pb, eb, tmp));
        double dE = isfinite(prevE) ? fabs(E[5] - prevE) : INFINITY;
        conv = dE < 1.0e-11 && effd < 1.0e-9 && resid < 1.0e-7;
        if (!conv) {
            memcpy(prev_a, pa, B * na_);
            if (!closed) memcpy(prev_b, pb, B * nb_);
        }
        if (conv) break;
        if (isfinite(prevD)) {
            if (effd > prevD * 1.05) mixing = maxd(0.10, mixing * 0.75);
            else if (effd < prevD) mixing = mind(0.50, mixing * 1.10);
        }
        for (long p = 0; p < N; ++p) {
            da[p] = (1.0 - imix) * da[p] + imix * oa[p];
            db[p] = (1.0 - imix) * db[p] + imix * ob[p];
        }
        prevD = effd;
        prevE = E[5];
    }
    const int done_it = it > max_it ? max_it : it;
    if (!rc) {
        for (int q = 0; q < 6; ++q) energies6[q] = E[q];
        stats4[0] = done_it;
        stats4[1] = conv ? 1.0 : 0.0;
        stats4[2] = effd;
        stats4[3] = resid;
        int k = 0;
        for (int i = 0; i < na_ && k < n_eig; ++i) eig_out[k++] = ea[i];
        for (int i = 0; i < nb_ && k < n_eig; ++i) eig_out[k++] = eb[i];
        if (dens_out) {
            memcpy(dens_out, oa, B);
            memcpy(dens_out + N, ob, B);
        }
    }
    if (seconds2) {
        seconds2[0] = t_init - t_begin;
        seconds2[1] = (now_s() - t_init) / (done_it > 0 ? done_it : 1);
    }
    free(vext); free(da); free(db); free(rho); free(vh); free(vxa); free(vxb); free(va); free(vb);
    free(oa); free(ob); free(orho); free(ovh); free(tmp); free(pall); free(prev_a); free(prev_b);
    free(ea); free(eb); free(ones);
    return rc;
}

int oracle_scf_molecule(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int charge,
                        int multiplicity, int kind, double* energies6, double* stats4, int n_eig, double* eig_out,
                        double* dens_out) {
    return scf_run(n, b, nnuc, Z, xyz, charge, multiplicity, kind, energies6, stats4, n_eig, eig_out, dens_out, 250,
                   NULL);
}

/* CPU-baseline sample: initial densities, then `iterations` SCF iterations of the loop above
 * (the reference's algorithm); seconds2 = {initialisation, mean seconds per iteration}. */
int oracle_scf_sample(const long* n, const double* b, int nnuc, const int* Z, const double* xyz, int multiplicity,
                      int kind, int iterations, double* seconds2) {
    double e6[6], st[4], eig[1024];
    return scf_run(n, b, nnuc, Z, xyz, 0, multiplicity, kind, e6, st, 1024, eig, NULL, iterations, seconds2);
}


/* ======================================================== radial path ====== */
/* RadialGrid.cpp:5-21: r_i = (i+1) * rMax/(points+1).  Every radial routine of the
 * reference takes its step as r[1]-r[0]; so does this restatement. */
typedef struct {
    long n;
    double* r;
    double dr; /* r[1] - r[0] */
} rgrid;

static int make_rgrid(long points, double rmax, rgrid* g) {
    if (points == 0) FAIL("El numero de puntos debe ser mayor que cero.");
    if (rmax <= 0.0) FAIL("RMAX debe ser mayor que cero.");
    double h = rmax / (double)(points + 1);
    g->n = points;
    g->r = malloc(sizeof(double) * (size_t)points);
    for (long i = 0; i < points; ++i) g->r[i] = (double)(i + 1) * h;
    g->dr = points > 1 ? g->r[1] - g->r[0] : h;
    return 0;
}

/* buildKohnShamHamiltonian, KohnShamHamiltonian.cpp:6-101: diag and the constant off-diagonal */
static void radial_h(const rgrid* g, const double* veff, int l, double* diag, double* off) {
    double idr2 = 1.0 / (g->dr * g->dr);
    double cc = 0.5 * (double)(l * (l + 1));
    for (long i = 0; i < g->n; ++i) diag[i] = idr2 + cc / (g->r[i] * g->r[i]) + veff[i];
    *off = -0.5 * idr2;
}

static double eps_guard(double v) { return fabs(v) < EPS_ ? copysign(EPS_, v == 0.0 ? 1.0 : v) : v; }

/* countEigenvaluesBelow + sturmPivot, EigenvalueSolver.cpp:13-92 (off-diagonals all equal) */
static long sturm_count(long n, const double* diag, double off, double E) {
    long c = 0;
    double prev = diag[0] - E;
    if (prev < 0.0) ++c;
    prev = eps_guard(prev);
    double oo = off * off;
    for (long i = 1; i < n; ++i) {
        double piv = diag[i] - E - oo / eps_guard(prev);
        if (piv < 0.0) ++c;
        prev = eps_guard(piv);
    }
    return c;
}

/* findEigenvalue, EigenvalueSolver.cpp:94-221 */
static int find_eigenvalue(long n, const double* diag, double off, long index, double lo, double hi, double* out) {
    long lc = sturm_count(n, diag, off, lo), hc = sturm_count(n, diag, off, hi);
    double w = hi - lo;
    for (int e = 0; e < 100; ++e) {
        if (lc <= index && index < hc) break;
        w *= 2.0;
        if (lc > index) {
            lo -= w;
            lc = sturm_count(n, diag, off, lo);
        }
        if (hc <= index) {
            hi += w;
            hc = sturm_count(n, diag, off, hi);
        }
    }
    if (lc > index || index >= hc) FAIL("No se pudo acotar el autovalor solicitado.");
    for (int it = 0; it < 300; ++it) {
        double mid = 0.5 * (lo + hi);
        long c = sturm_count(n, diag, off, mid);
        if (c <= index) lo = mid;
        else hi = mid;
        double tol = 1.0e-13 * maxd(1.0, maxd(fabs(lo), fabs(hi)));
        if (hi - lo <= tol) break;
    }
    *out = 0.5 * (lo + hi);
    return 0;
}

/* solveTridiagonal (Thomas), NumericalMethods.cpp:85-139, constant off-diagonals */
static int thomas(long n, const double* diag0, double off, const double* rhs, double* sol, double* dwork) {
    memcpy(dwork, diag0, sizeof(double) * (size_t)n);
    memcpy(sol, rhs, sizeof(double) * (size_t)n);
    for (long i = 1; i < n; ++i) {
        if (fabs(dwork[i - 1]) < EPS_) FAIL("Pivote numericamente singular en el solver tridiagonal.");
        double f = off / dwork[i - 1];
        dwork[i] -= f * off;
        sol[i] -= f * sol[i - 1];
    }
    if (fabs(dwork[n - 1]) < EPS_) FAIL("Pivote final numericamente singular en el solver tridiagonal.");
    sol[n - 1] /= dwork[n - 1];
    for (long i = n - 1; i-- > 0;) {
        if (fabs(dwork[i]) < EPS_) FAIL("Pivote numericamente singular en el solver tridiagonal.");
        sol[i] = (sol[i] - off * sol[i + 1]) / dwork[i];
    }
    return 0;
}

/* solveEigenvector (inverse iteration), EigenvalueSolver.cpp:223-321 */
static int inverse_iteration(long n, const double* diag, double off, double E, double* vec) {
    double* sh = malloc(sizeof(double) * (size_t)n);
    double* nx = malloc(sizeof(double) * (size_t)n);
    double* wk = malloc(sizeof(double) * (size_t)n);
    int rc = 0;
    for (long i = 0; i < n; ++i) vec[i] = sin((double)(i + 1));
    double nn = sqrt(vdot(n, vec, vec));
    if (nn < EPS_) { free(sh); free(nx); free(wk); FAIL("Vector inicial numericamente nulo."); }
    for (long i = 0; i < n; ++i) vec[i] /= nn;
    double shift = E + 1.0e-10 * maxd(1.0, fabs(E));
    for (long i = 0; i < n; ++i) sh[i] = diag[i] - shift;
    for (int it = 0; it < 1000; ++it) {
        if ((rc = thomas(n, sh, off, vec, nx, wk))) break;
        double m = sqrt(vdot(n, nx, nx));
        if (m < EPS_) { snprintf(g_err, sizeof g_err, "Autovector numericamente nulo."); rc = 1; break; }
        for (long i = 0; i < n; ++i) nx[i] /= m;
        if (vdot(n, vec, nx) < 0.0)
            for (long i = 0; i < n; ++i) nx[i] = -nx[i];
        double d = 0.0;
        for (long i = 0; i < n; ++i) d = maxd(d, fabs(vec[i] - nx[i]));
        memcpy(vec, nx, sizeof(double) * (size_t)n);
        if (d < 1.0e-12) break;
    }
    free(sh); free(nx); free(wk);
    return rc;
}

/* normalizeVector, NumericalMethods.cpp:34-61 */
static int rnormalize(long n, double* v, double dr) {
    double nn = sqrt(dr * vdot(n, v, v));
    if (nn < EPS_) FAIL("No se puede normalizar un vector con norma cero.");
    for (long i = 0; i < n; ++i) v[i] /= nn;
    return 0;
}

/* solveOrbital, EigenvalueSolver.cpp:323-404 */
static int radial_orbital(const rgrid* g, const double* diag, double off, long index, double* eig, double* u) {
    double mn = diag[0], mx = diag[0];
    for (long i = 1; i < g->n; ++i) {
        mn = mind(mn, diag[i]);
        mx = maxd(mx, diag[i]);
    }
    TRY(find_eigenvalue(g->n, diag, off, index, mn - 10.0, mx + 10.0, eig));
    TRY(inverse_iteration(g->n, diag, off, *eig, u));
    return rnormalize(g->n, u, g->dr);
}

int oracle_radial_solve_orbital(long points, double rmax, const double* veff, int l, int index, double* eig,
                                double* u_out) {
    rgrid g;
    TRY(make_rgrid(points, rmax, &g));
    double* d = malloc(sizeof(double) * (size_t)points);
    double off;
    radial_h(&g, veff, l, d, &off);
    int rc = radial_orbital(&g, d, off, index, eig, u_out);
    free(d);
    free(g.r);
    return rc;
}

int oracle_radial_sturm_count(long points, double rmax, const double* veff, int l, double energy, long* count) {
    rgrid g;
    TRY(make_rgrid(points, rmax, &g));
    double* d = malloc(sizeof(double) * (size_t)points);
    double off;
    radial_h(&g, veff, l, d, &off);
    *count = sturm_count(points, d, off, energy);
    free(d);
    free(g.r);
    return 0;
}

/* calculateHartreePotential (radial), HartreePotential.cpp:8-86 */
static void radial_hartree(const rgrid* g, const double* rho, double* v, double* enc, double* outer) {
    const double* r = g->r;
    long n = g->n;
    double dr = g->dr;
    enc[0] = 0.0;
    for (long i = 1; i < n; ++i) {
        double f0 = 4.0 * PI_ * r[i - 1] * r[i - 1] * rho[i - 1];
        double f1 = 4.0 * PI_ * r[i] * r[i] * rho[i];
        enc[i] = enc[i - 1] + 0.5 * (f0 + f1) * dr;
    }
    outer[n - 1] = 0.0;
    for (long i = n - 1; i-- > 0;) {
        double f0 = 4.0 * PI_ * r[i] * rho[i];
        double f1 = 4.0 * PI_ * r[i + 1] * rho[i + 1];
        outer[i] = outer[i + 1] + 0.5 * (f0 + f1) * dr;
    }
    for (long i = 0; i < n; ++i) v[i] = enc[i] / r[i] + outer[i];
}

int oracle_radial_hartree(long points, double rmax, const double* rho, double* out) {
    rgrid g;
    TRY(make_rgrid(points, rmax, &g));
    if (points < 2) FAIL("Se necesitan al menos dos puntos radiales.");
    double* a = malloc(sizeof(double) * (size_t)points);
    double* c = malloc(sizeof(double) * (size_t)points);
    radial_hartree(&g, rho, out, a, c);
    free(a); free(c); free(g.r);
    return 0;
}

/* calculateRadialGradient, ExchangeCorrelation.cpp:10-51 */
static double rgrad(const rgrid* g, const double* f, long i) {
    const double* r = g->r;
    long n = g->n;
    if (i == 0) return (f[1] - f[0]) / (r[1] - r[0]);
    if (i == n - 1) return (f[n - 1] - f[n - 2]) / (r[n - 1] - r[n - 2]);
    return (f[i + 1] - f[i - 1]) / (r[i + 1] - r[i - 1]);
}

/* calculateRadialDivergence, ExchangeCorrelation.cpp:53-150 */
static double rdiv(const rgrid* g, const double* c, long i) {
    const double* r = g->r;
    long n = g->n;
    if (r[i] == 0.0) return 0.0;
    if (i == 0) return ((r[1] * r[1] * c[1] - r[0] * r[0] * c[0]) / (r[1] - r[0])) / (r[0] * r[0]);
    if (i == n - 1)
        return ((r[n - 1] * r[n - 1] * c[n - 1] - r[n - 2] * r[n - 2] * c[n - 2]) / (r[n - 1] - r[n - 2])) /
               (r[n - 1] * r[n - 1]);
    return ((r[i + 1] * r[i + 1] * c[i + 1] - r[i - 1] * r[i - 1] * c[i - 1]) / (r[i + 1] - r[i - 1])) / (r[i] * r[i]);
}

/* calculateSpinExchangeCorrelationPotential, ExchangeCorrelation.cpp:154-274 */
static void radial_xc_pot(int kind, const rgrid* g, const double* na, const double* nb, int spin, double* out,
                          double* dd, double* cc) {
    for (long i = 0; i < g->n; ++i) {
        double r5[5];
        xc_eval(kind, na[i], nb[i], rgrad(g, na, i), rgrad(g, nb, i), r5);
        dd[i] = spin == 0 ? r5[1] : r5[2];
        cc[i] = spin == 0 ? r5[3] : r5[4];
    }
    for (long i = 0; i < g->n; ++i) {
        if (na[i] + nb[i] <= RHO_FLOOR_) {
            out[i] = 0.0;
            continue;
        }
        if (g->r[i] == 0.0) {
            out[i] = dd[i];
            continue;
        }
        out[i] = dd[i] - rdiv(g, cc, i);
    }
}

int oracle_radial_xc_potential(int kind, long points, double rmax, const double* na, const double* nb, int spin,
                               double* out) {
    rgrid g;
    TRY(make_rgrid(points, rmax, &g));
    if (spin != 0 && spin != 1) FAIL("El canal de spin debe ser 0 (alpha) o 1 (beta).");
    double* a = malloc(sizeof(double) * (size_t)points);
    double* c = malloc(sizeof(double) * (size_t)points);
    radial_xc_pot(kind, &g, na, nb, spin, out, a, c);
    free(a); free(c); free(g.r);
    return 0;
}

/* calculateSpinExchangeCorrelationEnergy, ExchangeCorrelation.cpp:276-371 */
static double radial_xc_en(int kind, const rgrid* g, const double* na, const double* nb) {
    double e = 0.0;
    for (long i = 0; i < g->n; ++i) {
        double n = na[i] + nb[i], ex = 0.0;
        if (n > RHO_FLOOR_) {
            double r5[5];
            xc_eval(kind, na[i], nb[i], rgrad(g, na, i), rgrad(g, nb, i), r5);
            ex = r5[0];
        }
        double in = 4.0 * PI_ * g->r[i] * g->r[i] * n * ex;
        if (i == 0 || i == g->n - 1) e += 0.5 * in;
        else e += in;
    }
    return e * g->dr;
}

int oracle_radial_xc_energy(int kind, long points, double rmax, const double* na, const double* nb, double* e) {
    rgrid g;
    TRY(make_rgrid(points, rmax, &g));
    *e = radial_xc_en(kind, &g, na, nb);
    free(g.r);
    return 0;
}

/* getAtomicConfiguration + buildStates, ElectronicConfiguration.cpp:16-146 */
int oracle_atomic_configuration(int Z, int cap, int* rows, int* nrows) {
    if (Z < 1 || Z > 30) FAIL("Configuracion atomica no disponible para Z = %d", Z);
    int sh[8][3], k = 0;
    sh[k][0] = 1; sh[k][1] = 0; sh[k][2] = Z < 2 ? Z : 2; ++k;
    if (Z >= 3) { sh[k][0] = 2; sh[k][1] = 0; sh[k][2] = (Z - 2) < 2 ? Z - 2 : 2; ++k; }
    if (Z >= 5) { sh[k][0] = 2; sh[k][1] = 1; sh[k][2] = (Z - 4) < 6 ? Z - 4 : 6; ++k; }
    if (Z >= 11) { sh[k][0] = 3; sh[k][1] = 0; sh[k][2] = (Z - 10) < 2 ? Z - 10 : 2; ++k; }
    if (Z >= 13) { sh[k][0] = 3; sh[k][1] = 1; sh[k][2] = (Z - 12) < 6 ? Z - 12 : 6; ++k; }
    if (Z >= 19) {
        int s = Z >= 20 ? 2 : 1;
        if (Z == 24 || Z == 29) s = 1;
        sh[k][0] = 4; sh[k][1] = 0; sh[k][2] = s; ++k;
    }
    if (Z >= 21) {
        int d = Z - 20;
        if (Z == 24) d = 5;
        else if (Z >= 29) d = 10;
        sh[k][0] = 3; sh[k][1] = 2; sh[k][2] = d; ++k;
    }
    for (int q = 0; q < k && q < cap; ++q) {
        int capacity = 2 * sh[q][1] + 1;
        int a = sh[q][2] < capacity ? sh[q][2] : capacity;
        rows[4 * q + 0] = sh[q][0];
        rows[4 * q + 1] = sh[q][1];
        rows[4 * q + 2] = a;
        rows[4 * q + 3] = sh[q][2] - a;
    }
    *nrows = k;
    return 0;
}

/* One occupied radial orbital: {n, l, spin, electrons, eigenvalue, u}. */
typedef struct {
    int n, l, spin, el;
    double eig;
    double* u;
} rorb;

/* calculateSpinDensity, ElectronDensity.cpp:8-56 */
static void radial_density(const rgrid* g, const rorb* o, int no, int spin, double* d) {
    for (long i = 0; i < g->n; ++i) d[i] = 0.0;
    for (int q = 0; q < no; ++q) {
        if (o[q].spin != spin || o[q].el <= 0) continue;
        for (long i = 0; i < g->n; ++i) d[i] += (double)o[q].el * o[q].u[i] * o[q].u[i] / (4.0 * PI_ * g->r[i] * g->r[i]);
    }
}

/* calculateDensityDifference, SelfConsistentField.cpp:414-485 */
static double radial_ddiff(const rgrid* g, const double* o, const double* nw) {
    double d2 = 0.0, n2 = 0.0;
    for (long i = 0; i < g->n; ++i) {
        double w = 4.0 * PI_ * g->r[i] * g->r[i];
        double d = nw[i] - o[i];
        d2 += d * d * w;
        n2 += nw[i] * nw[i] * w;
    }
    double dn = sqrt(d2 * g->dr), nn = sqrt(n2 * g->dr);
    if (nn <= EPS_) return dn;
    return dn / nn;
}

/* solveSelfConsistentField, SelfConsistentField.cpp:539-786 with solveSpinOrbitals (:28-77),
 * calculateMaximumKSResidual (:110-205), buildInitialSpinOrbitals (:207-308),
 * buildEffectivePotentials (:341-412), calculateTotalEnergy (TotalEnergy.cpp:170-242). */
int oracle_solve_atom(int Z, int kind, long points, double rmax, double* energies5, double* stats4, int n_eig,
                      double* eig_out, int* n_eig_written) {
    rgrid g;
    TRY(make_rgrid(points, rmax, &g));
    if (points < 2) FAIL("La malla radial debe contener al menos dos puntos.");
    int rows[64], nr;
    TRY(oracle_atomic_configuration(Z, 16, rows, &nr));
    const long n = g.n;
    const double* r = g.r;
    size_t B = sizeof(double) * (size_t)n;
    rorb orb[32];
    int no = 0;
    /* orbital list in the reference order: alpha states, then beta states */
    for (int s = 0; s < 2; ++s)
        for (int q = 0; q < nr; ++q) {
            int el = rows[4 * q + 2 + s];
            if (el <= 0) continue;
            orb[no].n = rows[4 * q];
            orb[no].l = rows[4 * q + 1];
            orb[no].spin = s;
            orb[no].el = el;
            orb[no].eig = 0.0;
            orb[no].u = malloc(B);
            ++no;
        }
    double *da = malloc(B), *db = malloc(B), *va = malloc(B), *vb = malloc(B), *vh = malloc(B);
    double *oa = malloc(B), *ob = malloc(B), *od = malloc(B), *rd = malloc(B), *diag = malloc(B);
    double *w1 = malloc(B), *w2 = malloc(B);
    int rc = 0;
    /* buildInitialSpinOrbitals :207-308: hydrogenic r^{l+1} e^{-max(0.15, Z/n^2) r}, per spin in state
     * order (which is the same order as the orbital list above) */
    for (int q = 0; q < no && !rc; ++q) {
        double ex = maxd(0.15, (double)Z / ((double)orb[q].n * (double)orb[q].n));
        for (long i = 0; i < n; ++i) orb[q].u[i] = pow(r[i], (double)(orb[q].l + 1)) * exp(-ex * r[i]);
        rc = rnormalize(n, orb[q].u, g.dr);
    }
    if (!rc) {
        radial_density(&g, orb, no, 0, da);
        radial_density(&g, orb, no, 1, db);
    }
    double prevE = INFINITY, prevD = INFINITY, mixing = 0.25;
    double E[5] = {0}, effd = 0.0, resid = 0.0;
    int it, conv = 0;
    double idr2 = 1.0 / (g.dr * g.dr);
    for (it = 1; !rc && it <= 250; ++it) {
        /* buildEffectivePotentials :341-412 */
        for (long i = 0; i < n; ++i) rd[i] = da[i] + db[i];
        radial_hartree(&g, rd, vh, w1, w2);
        radial_xc_pot(kind, &g, da, db, 0, va, w1, w2);
        radial_xc_pot(kind, &g, da, db, 1, vb, w1, w2);
        for (long i = 0; i < n; ++i) {
            double nuc = -(double)Z / r[i];
            va[i] += nuc + vh[i];
            vb[i] += nuc + vh[i];
        }
        /* solveAllSpinOrbitals :79-108; the eigen-index counts same-spin states per l (:56-57) */
        for (int s = 0; s < 2 && !rc; ++s) {
            int count_l[4] = {0, 0, 0, 0};
            for (int q = 0; q < no && !rc; ++q) {
                if (orb[q].spin != s) continue;
                double off;
                radial_h(&g, s == 0 ? va : vb, orb[q].l, diag, &off);
                rc = radial_orbital(&g, diag, off, count_l[orb[q].l]++, &orb[q].eig, orb[q].u);
            }
        }
        if (rc) break;
        radial_density(&g, orb, no, 0, oa);
        radial_density(&g, orb, no, 1, ob);
        for (long i = 0; i < n; ++i) {
            rd[i] = da[i] + db[i];
            od[i] = oa[i] + ob[i];
        }
        radial_hartree(&g, od, vh, w1, w2);
        /* calculateKineticEnergy, TotalEnergy.cpp:10-101 */
        double T = 0.0;
        for (int q = 0; q < no; ++q) {
            double cc = 0.5 * (double)(orb[q].l * (orb[q].l + 1)), oe = 0.0, kod = -0.5 * idr2;
            const double* u = orb[q].u;
            for (long i = 0; i < n; ++i) {
                double ap = (idr2 + cc / (r[i] * r[i])) * u[i];
                if (i > 0) ap += kod * u[i - 1];
                if (i + 1 < n) ap += kod * u[i + 1];
                oe += u[i] * ap;
            }
            T += (double)orb[q].el * oe * g.dr;
        }
        /* calculateExternalEnergy :103-168, calculateHartreeEnergy HartreePotential.cpp:88-137 */
        double ee = 0.0, eh = 0.0;
        for (long i = 0; i < n; ++i) {
            double in = -(double)Z * 4.0 * PI_ * r[i] * od[i];
            double ih = 4.0 * PI_ * r[i] * r[i] * od[i] * vh[i];
            if (i == 0 || i == n - 1) {
                ee += 0.5 * in;
                eh += 0.5 * ih;
            } else {
                ee += in;
                eh += ih;
            }
        }
        ee *= g.dr;
        eh = 0.5 * eh * g.dr;
        double exc = radial_xc_en(kind, &g, oa, ob);
        E[0] = T; E[1] = ee; E[2] = eh; E[3] = exc;
        E[4] = T + ee + eh + exc;
        double dd = radial_ddiff(&g, rd, od);
        double sdd = maxd(radial_ddiff(&g, da, oa), radial_ddiff(&g, db, ob));
        effd = maxd(dd, sdd);
        double dE = isfinite(prevE) ? fabs(E[4] - prevE) : INFINITY;
        /* calculateMaximumKSResidual :110-205 */
        resid = 0.0;
        for (int q = 0; q < no; ++q) {
            double off;
            radial_h(&g, orb[q].spin == 0 ? va : vb, orb[q].l, diag, &off);
            const double* u = orb[q].u;
            double s2 = 0.0;
            for (long i = 0; i < n; ++i) {
                double v = diag[i] * u[i];
                if (i > 0) v += off * u[i - 1];
                if (i + 1 < n) v += off * u[i + 1];
                double rr = v - orb[q].eig * u[i];
                s2 += rr * rr;
            }
            resid = maxd(resid, sqrt(s2 * g.dr));
        }
        if (effd < 1.0e-9 && dE < 1.0e-11 && resid < 1.0e-7) {
            conv = 1;
            break;
        }
        if (isfinite(prevD)) {
            if (effd > prevD * 1.05) mixing = maxd(0.10, mixing * 0.50);
            else if (effd < prevD) mixing = mind(0.50, mixing * 1.10);
        }
        for (long i = 0; i < n; ++i) {
            da[i] = (1.0 - mixing) * da[i] + mixing * oa[i];
            db[i] = (1.0 - mixing) * db[i] + mixing * ob[i];
        }
        prevD = effd;
        prevE = E[4];
    }
    if (!rc) {
        for (int q = 0; q < 5; ++q) energies5[q] = E[q];
        stats4[0] = it > 250 ? 250 : it;
        stats4[1] = conv ? 1.0 : 0.0;
        stats4[2] = effd;
        stats4[3] = resid;
        int k = 0;
        for (int q = 0; q < no && k < n_eig; ++q) eig_out[k++] = orb[q].eig;
        *n_eig_written = k;
    }
    for (int q = 0; q < no; ++q) free(orb[q].u);
    free(da); free(db); free(va); free(vb); free(vh); free(oa); free(ob); free(od); free(rd); free(diag);
    free(w1); free(w2); free(g.r);
    return rc;
}
