// Pointwise exchange-correlation functionals, callable from device code.
//
//  PZ81  — Slater exchange with spin scaling + Perdew–Zunger 1981 correlation
//          (reference PZ81.cpp:11-501).
//  PBE96 — PBE exchange through the spin-scaling relation E_x[na,nb] = (E_x[2na]+E_x[2nb])/2
//          and PBE correlation on PW92 (reference PBE96.cpp:22-966).
//
// Both return {eps_xc, v_alpha, v_beta, c_alpha, c_beta} where c = d f / d(grad n_sigma) with
// the reference's sign convention, and honour its 1e-20 density floor.  The formulas,
// constants and branch points are the reference's (they define the functional); the
// expression order follows it so results agree to a few ulp (device libm vs glibc).
#pragma once

namespace dftb {
namespace xcf {

constexpr double PI = 3.141592653589793238462643383279502884;
constexpr double RHO_FLOOR = 1.0e-20;

struct Result {
    double eps, va, vb, ca, cb;
};

__host__ __device__ __forceinline__ double clamp1(double z) { return z < -1.0 ? -1.0 : (z > 1.0 ? 1.0 : z); }
__host__ __device__ __forceinline__ double sign_of(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }

// ------------------------------------------------------------------ PZ81 ------------
struct PZPar {
    double A, B, C, D, gamma, beta1, beta2;
};
// unpolarised / polarised parameter sets (PZ81.cpp:21-39)
__host__ __device__ __forceinline__ PZPar pz_unpol() { return {0.0311, -0.0480, 0.0020, -0.0116, -0.1423, 1.0529, 0.3334}; }
__host__ __device__ __forceinline__ PZPar pz_pol() { return {0.01555, -0.0269, 0.0007, -0.0048, -0.0843, 1.3981, 0.2611}; }

// eps_c(rs) and d eps_c / d rs for one parameter set (PZ81.cpp:52-120)
__host__ __device__ __forceinline__ void pz_corr(double rs, double lrs, double srs, const PZPar& p, double& e,
                                                 double& de) {
    if (rs < 1.0) {
        e = p.A * lrs + p.B + p.C * rs * lrs + p.D * rs;
        de = p.A / rs + p.C * (lrs + 1.0) + p.D;
    } else {
        const double den = 1.0 + p.beta1 * srs + p.beta2 * rs;
        e = p.gamma / den;
        const double dden = p.beta1 / (2.0 * srs) + p.beta2;
        de = -p.gamma * dden / (den * den);
    }
}

__host__ __device__ inline Result pz81(double na_in, double nb_in) {
    Result r{0.0, 0.0, 0.0, 0.0, 0.0};
    const double a = na_in > 0.0 ? na_in : 0.0;
    const double b = nb_in > 0.0 ? nb_in : 0.0;
    const double n = a + b;
    if (n <= RHO_FLOOR) return r;
    const double z = clamp1((a - b) / n);
    const double rs = cbrt(3.0 / (4.0 * PI * n));
    // rs < 1 branch needs log(rs); rs >= 1 needs sqrt(rs)
    const double lrs = rs < 1.0 ? log(rs) : 0.0;
    const double srs = rs < 1.0 ? 0.0 : sqrt(rs);
    const double opz = 1.0 + z, omz = 1.0 - z;
    const double p43a = pow(opz, 4.0 / 3.0), p43b = pow(omz, 4.0 / 3.0);
    const double fden = pow(2.0, 4.0 / 3.0) - 2.0;
    const double f = (p43a + p43b - 2.0) / fden;                               // PZ81.cpp:122-149
    const double df = 4.0 / 3.0 * (pow(opz, 1.0 / 3.0) - pow(omz, 1.0 / 3.0)) / fden;  // :151-182
    const double ex = -0.7385587663820223 * cbrt(n);                             // :184-190
    const double sx = (p43a + p43b) / 2.0;                                      // :192-213
    const double dsx = 2.0 / 3.0 * (pow(opz, 1.0 / 3.0) - pow(omz, 1.0 / 3.0)); // :215-237
    double e0, d0, e1, d1;
    pz_corr(rs, lrs, srs, pz_unpol(), e0, d0);
    pz_corr(rs, lrs, srs, pz_pol(), e1, d1);
    const double exs = ex * sx;
    const double ec = e0 + f * (e1 - e0);
    r.eps = exs + ec;                                                           // :252-291
    // potentials (:293-433)
    const double dexrs = -exs / rs;
    const double decrs = d0 + f * (d1 - d0);
    const double exc = exs + ec;
    const double dxcrs = dexrs + decrs;
    const double dxcz = ex * dsx + df * (e1 - e0);
    const double radial = exc - rs * dxcrs / 3.0;
    r.va = radial + (1.0 - z) * dxcz;
    r.vb = radial - (1.0 + z) * dxcz;
    return r;
}

// ------------------------------------------------------------------ PBE96 -----------
constexpr double THIRD = 1.0 / 3.0;
constexpr double FOUR_THIRDS = 4.0 / 3.0;
constexpr double TWO_THIRDS = 2.0 / 3.0;
constexpr double KAPPA = 0.804;
constexpr double MU = 0.2195149727645171;
constexpr double GAMMA = 0.031090690869654895;
constexpr double BETA = 0.06672455060314922;
constexpr double DELTA = BETA / GAMMA;
constexpr double SPIN_GAMMA = 0.51984209978974632953;
constexpr double SPIN_FZZ = 8.0 / (9.0 * SPIN_GAMMA);
constexpr double ETA = 1.0e-12;
constexpr double EXCHANGE_A = -0.73855876638202240588;
constexpr double KF_COEFFICIENT = 3.09366772628014;

// PW92 G(rs) in the gcor2 form and its rs derivative (PBE96.cpp:99-179)
__host__ __device__ __forceinline__ double gcor2(double a, double a1, double b1, double b2, double b3, double b4,
                                                 double srs, double& drs) {
    const double srs2 = srs * srs;
    const double q0 = -2.0 * a * (1.0 + a1 * srs2);
    const double q1 = 2.0 * a * srs * (b1 + srs * (b2 + srs * (b3 + b4 * srs)));
    const double q2 = log(1.0 + 1.0 / q1);
    const double q3 = a * (b1 / srs + 2.0 * b2 + srs * (3.0 * b3 + 4.0 * b4 * srs));
    drs = -2.0 * a * a1 * q2 - q0 * q3 / (q1 * (1.0 + q1));
    return q0 * q2;
}

// PBE exchange for one spin-scaled density: energy density, d/drho, d/d|g| (PBE96.cpp:347-444)
__host__ __device__ __forceinline__ void pbe_exchange(double rho, double g, double& ed, double& dn, double& dg) {
    ed = dn = dg = 0.0;
    if (rho <= 0.0) return;
    const double r13 = cbrt(rho);
    const double exu = EXCHANGE_A * r13;
    const double kf = KF_COEFFICIENT * r13;
    const double den = 2.0 * kf * rho;
    const double s = den > 0.0 ? g / den : 0.0;
    const double s2 = s * s;
    const double mk = MU / KAPPA;
    const double p0 = 1.0 + mk * s2;
    const double fx = 1.0 + KAPPA - KAPPA / p0;
    const double fs = 2.0 * KAPPA * mk / (p0 * p0);
    dn = exu * FOUR_THIRDS * (fx - s2 * fs);
    if (g > 0.0) dg = EXCHANGE_A * 0.161620459673995 * s * fs;
    ed = rho * exu * fx;
}

// PBE correlation: eps_c, v_a, v_b, d/d|g| (PBE96.cpp:446-810; PW92 :181-345)
__host__ __device__ __forceinline__ void pbe_correlation(double na, double nb, double ga, double gb, double& eps,
                                                         double& va, double& vb, double& dg) {
    eps = va = vb = dg = 0.0;
    const double n = na + nb;
    if (n <= 0.0) return;
    const double z = clamp1((na - nb) / n);
    const double gm = fabs(ga + gb);
    const double kf = cbrt(3.0 * PI * PI * n);
    const double rs = cbrt(3.0 / (4.0 * PI * n));
    const double opz = 1.0 + z, omz = 1.0 - z;
    const double phi = 0.5 * (pow(opz, TWO_THIRDS) + pow(omz, TWO_THIRDS));
    const double ks = sqrt(4.0 * kf / PI);
    const double tkp = 2.0 * ks * phi;
    const double t = tkp > 0.0 ? gm / (tkp * n) : 0.0;
    // PW92
    const double srs = sqrt(rs);
    double eud, epd, ad;
    const double eu = gcor2(0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, srs, eud);
    const double ep = gcor2(0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517, srs, epd);
    const double al = gcor2(0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671, srs, ad);
    const double z4 = z * z * z * z;
    const double f = (pow(opz, FOUR_THIRDS) + pow(omz, FOUR_THIRDS) - 2.0) / SPIN_GAMMA;
    const double ec = eu * (1.0 - f * z4) + ep * f * z4 - al * f * (1.0 - z4) / SPIN_FZZ;
    const double ecrs = eud * (1.0 - f * z4) + epd * f * z4 - ad * f * (1.0 - z4) / SPIN_FZZ;
    const double fz = FOUR_THIRDS * (pow(opz, THIRD) - pow(omz, THIRD)) / SPIN_GAMMA;
    const double ecz = 4.0 * z * z * z * f * (ep - eu + al / SPIN_FZZ) +
                       fz * (z4 * ep - z4 * eu - (1.0 - z4) * al / SPIN_FZZ);
    // H(t)
    const double phi3 = phi * phi * phi, phi4 = phi3 * phi;
    const double ex = -ec / (GAMMA * phi3);
    const double b = ex < 700.0 ? DELTA / expm1(ex) : DELTA * exp(-ex);
    const double b2 = b * b, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
    const double q4 = 1.0 + b * t2;
    const double q5 = 1.0 + b * t2 + b2 * t4;
    const double h = phi3 * (BETA / DELTA) * log(1.0 + DELTA * q4 * t2 / q5);
    const double fac = DELTA / b + 1.0;
    const double bec = b2 * fac / (BETA * phi3);
    const double q8 = q5 * q5 + DELTA * q4 * q5 * t2;
    const double q9 = 1.0 + 2.0 * b * t2;
    const double hb = -BETA * phi3 * b * t6 * (2.0 + b * t2) / q8;
    const double hrs = -(rs / 3.0) * hb * bec * ecrs;
    const double ht = 2.0 * BETA * phi3 * q9 / q8;
    const double comm = h + hrs - 7.0 * t2 * ht / 6.0;
    const double gz = (pow(opz + ETA, -THIRD) - pow(omz + ETA, -THIRD)) / 3.0;
    const double bg = -3.0 * b2 * ec * fac / (BETA * phi4);
    const double hz = 3.0 * gz * h / phi + hb * (bg * gz + bec * ecz);
    const double pref = hz - gz * t2 * ht / phi;
    const double common = ec - rs * ecrs / 3.0 - z * ecz;
    eps = ec + h;
    va = common + ecz + comm + pref * (1.0 - z);
    vb = common - ecz + comm + pref * (-1.0 - z);
    if (gm > 0.0) dg = t * ht / tkp;
}

__host__ __device__ inline Result pbe96(double na_in, double nb_in, double ga, double gb) {
    Result r{0.0, 0.0, 0.0, 0.0, 0.0};
    const double a = na_in > 0.0 ? na_in : 0.0;
    const double b = nb_in > 0.0 ? nb_in : 0.0;
    const double n = a + b;
    if (n <= RHO_FLOOR) return r;
    double eda, dna, dga, edb, dnb, dgb;
    pbe_exchange(2.0 * a, 2.0 * fabs(ga), eda, dna, dga);
    pbe_exchange(2.0 * b, 2.0 * fabs(gb), edb, dnb, dgb);
    double ec, vca, vcb, dgc;
    pbe_correlation(a, b, ga, gb, ec, vca, vcb, dgc);
    r.eps = 0.5 * (eda + edb) / n + ec;
    r.va = dna + vca;
    r.vb = dnb + vcb;
    const double cs = sign_of(ga + gb);
    r.ca = dga * sign_of(ga) + dgc * cs;
    r.cb = dgb * sign_of(gb) + dgc * cs;
    return r;
}

template <int KIND>
__host__ __device__ __forceinline__ Result evaluate(double na, double nb, double ga, double gb) {
    if (KIND == 1) return pbe96(na, nb, ga, gb);
    return pz81(na, nb);
}

}  // namespace xcf
}  // namespace dftb
