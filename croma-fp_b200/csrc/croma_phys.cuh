// croma_phys.cuh -- physics of CROMA's tracer Fokker-Planck update, shared
// by the host table builders and the sm_100a kernels.
//
// Formulas follow the reference (kosukenishiwaki/croma-fp) in its own
// evaluation order; each function names the file:line it restates.  Host
// instantiations run on glibc, device ones on CUDA's libm.  Quantities that
// depend only on the momentum grid (p^2, exp(-1/p), exp(-E/E_max), the
// Kamae cross section, the Coulomb kinematics) are evaluated once on the
// host and read by the kernels from GridTables, so the device reuses the
// reference's exact values for them.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define CROMA_HD __host__ __device__ __forceinline__
#else
#define CROMA_HD inline
#endif

namespace croma {

// Physical constants: src/CONSTANTS.c:3-19.
constexpr double kC = 2.999e+10;
constexpr double kGeV = 1.6e-3;
constexpr double kEV = 1.6e-12;
constexpr double kMsun = 1.99e+33;
constexpr double kMpc = 3.0857e+24;
constexpr double kKpc = 3.0857e+21;
constexpr double kGyr = 3.1536e+16;
constexpr double kHPlanck = 6.63e-27;
constexpr double kMp = 0.938;
constexpr double kMe = 0.511e-3;
constexpr double kMb = 1.0e-27;
constexpr double kMpiCh = 1.40e-1;
constexpr double kMmu = 1.05e-1;
constexpr double kPi = 3.14159265358979323846;
constexpr double kEpMax = 1.0e7;          // tracer_fp_coef.c:262

enum DppModel { kDppAsa = 1, kDppTtd = 2, kDppOff = 3, kDppDirect = 4 };

// Error bits raised by kernels into the context's device error word.
enum ErrBits : unsigned {
    kErrSingular = 1u,      // Thomas pivot |d| <= 1e-300 (fp_shared_core.c:235-245)
    kErrCcNan = 2u,         // NaN at the right CC boundary (Chang_Cooper.c:166-183)
    kErrIcNewton = 4u,      // CMB bound iteration did not converge
    kErrBadInput = 8u,
};

// Maximum bins per species supported by the kernels.
constexpr int kMaxNb = 512;

// Per-species grid tables (device pointers), built once per context.
struct SpeciesTables {
    const double *p, *dp, *E;
    const double *p2;           // p^2 (FP_Coef.c:97, 141)
    const double *exp_cut;      // exp(-1/p) (FP_Coef.c:98, 142)
    const double *two_over_p;   // 2/p used in B = radp - 2 Dpp / p (fp_shared_core.c:2401)
    const double *expE;         // exp(-E/E_max) (protons; FP_Coef.c:699)
    const double *inv_dx;       // 1 / dp
    const double *inv_dxl;      // 1 / (p[j] - p[j-1])   (j >= 1)
    const double *inv_dxr;      // 1 / (p[j+1] - p[j])   (j <= nb-2)
    const double *dxf;          // p[j+1] - p[j]         (j <= nb-2), face widths
    const double *face_rf;      // dxf[j] / (g[j] + g[j+1]), g = p^2 expE exp(-1/p) (j <= nb-2)
    double pm1, pp1;
    double pm1_p2, pp1_p2, pm1_exp_cut, pp1_exp_cut;
    double expE_m1, expE_p1;    // exp(-m_p sqrt(1+p^2)/E_max) at the ghost edges
};

struct GridTables {
    SpeciesTables s[2];         // 0 = proton, 1 = electron
    // proton Coulomb kinematics (b_Coulomb_p, FP_Coef.c:438-449)
    const double *cp_Ep;        // gamma m_p - m_p
    const double *cp_kin;       // gamma - 1
    const double *cp_inv_betap2;// 1 / (p^2/(1+p^2))
    double cpm1_Ep, cpm1_kin, cpm1_inv_betap2;
    double cpp1_Ep, cpp1_kin, cpp1_inv_betap2;
    const double *sig_eff;      // sigma_pp(max(j, j_pp)) * sigmoid (fp_shared_core.c:760-765)
    const double *cp_inv2mpkin; // 1 / (2 m_p (gamma - 1))
    // electron kinematics (prepare_cre_losses_1d, fp_shared_core.c:818-841)
    const double *ce_logp;      // log(p)
    const double *ce_beta2;     // p^2/(1+p^2)
    const double *ce_inv_beta2; // (1+p^2)/p^2
    double cem1_beta2, cep1_beta2;
    // secondary electrons (prepare_secondary_kernel_flat, transposed [jp][je])
    const double *fqe;
    int fqe_jp0;
    int nb;
};

// ----------------------------------------------------------------------
// Losses
// ----------------------------------------------------------------------
CROMA_HD double coulomb_kernel(double x)   // b_Coulomb_kernel, FP_Coef.c:451-453
{
    return 0.5 * sqrt(kPi) * erf(sqrt(x)) - sqrt(x) * exp(-x);
}

// The same kernel with its saturated tail taken exactly: for x > 40,
// erf(sqrt(x)) rounds to 1 (erfc(6.32) < 1e-18) and sqrt(x) exp(-x) < 3e-17
// is below half an ulp of 0.5 sqrt(pi), so the double result is exactly
// 0.5 sqrt(pi).
CROMA_HD double coulomb_kernel_fast(double x)
{
    if (x > 40.0) return 0.5 * sqrt(kPi);
    return 0.5 * sqrt(kPi) * erf(sqrt(x)) - sqrt(x) * exp(-x);
}

// b_Coulomb_p, FP_Coef.c:438-449, with the grid-only kinematics passed in.
CROMA_HD double coulomb_p(double n, double kbt, double Ep, double kinetic, double inv_betap2)
{
    const double xp = Ep / kbt;
    const double xe = xp * (kMe / kMp);
    const double sum = coulomb_kernel(xe) + coulomb_kernel(xp) * (kMe / kMp);
    const double thermal = 1.0 - kbt / (2.0 * kMp * kinetic);
    if (thermal < 0.0) return 0.0;
    return kGyr * kC / (kMp * kGeV) * sum * n * inv_betap2 * thermal * 3.5e-29;
}

// b_Coulomb_p from p, as the sub-step estimator calls it (tracer_fp_nsub.c:260-263).
CROMA_HD double coulomb_p_from_p(double n, double p, double kbt)
{
    const double p2 = p * p;
    const double gamma = sqrt(1.0 + p2);
    const double betap2 = p2 / (1.0 + p2);
    const double kinetic = gamma - 1.0;
    const double Ep = gamma * kMp - kMp;
    const double xp = Ep / kbt;
    const double xe = xp * (kMe / kMp);
    const double sum = coulomb_kernel(xe) + coulomb_kernel(xp) * (kMe / kMp);
    const double thermal = 1.0 - kbt / (2.0 * kMp * kinetic);
    if (thermal < 0.0) return 0.0;
    return kGyr * kC / (kMp * kGeV) * sum * n * (1.0 / betap2) * thermal * 3.5e-29;
}

CROMA_HD double b_synch(double p, double B)        // FP_Coef.c:454-462
{
    const double b_ratio = B * 1.0e+6 / 3.2;
    return 4.8e-4 * p * p * b_ratio * b_ratio * 9.11e-28 * 3.0e+10 * 3.1536e+16;
}

CROMA_HD double b_coulomb_e(double n, double pe)   // FP_Coef.c:464-469
{
    const double pe2 = pe * pe;
    const double beta2 = pe2 / (1.0 + pe2);
    return 3.05e-29 * n * (1.0 + log(pe / n) / 74.8) / (kMe * kGeV) * kC * kGyr / beta2;
}

// ----------------------------------------------------------------------
// Acceleration times (FP_Coef.c:624-678)
// ----------------------------------------------------------------------
CROMA_HD double i_theta(double x)
{
    return x * x * x * x / 4.0 + x * x - (1.0 + 2.0 * x * x) * log(x) - 5.0 / 4.0;
}

CROMA_HD double tacc_ttd(int model_brunetti16, double L, double cs, double Ms, double v)
{
    const double x = cs / kC;
    if (model_brunetti16) {
        const double theta = i_theta(x);
        if (!(x > 0.0) || !(theta > 0.0) || !(Ms > 0.0) || !(L > 0.0) || !(cs > 0.0)) return 0.0;
        const double r = Ms / 0.5;
        return 2.5e-3 / (x * theta) * (1.0 / (r * r * r * r)) * (L / (300.0 * kKpc)) *
               (1.0 / (cs / 1500.0e5));
    }
    const double kL = 2.0 * kPi / L;
    const double k_cut = 1.04e+4 * (Ms * Ms * Ms * Ms) * kL;
    const double kWk_L = 0.5 * (v * v);
    const double kWk_cut = kWk_L * (1.0 / sqrt(k_cut / kL));
    return kC / kPi / i_theta(x) / k_cut / kWk_cut / kGyr;
}

CROMA_HD double tacc_asa(double psi3, double L, double cs, double Ms, double beta_pl)
{
    return sqrt(6.0 / 5.0) / 12.0 * (kC / cs / cs) * L / sqrt(beta_pl) / (Ms * Ms * Ms) * psi3 / kGyr;
}

CROMA_HD double effective_mach(double mach_limit, double dv, double cs)
{
    if (cs <= 0.0) return 0.0;
    double m = dv / cs;
    if (m < 0.0) m = 0.0;
    if (mach_limit > 0.0 && m > mach_limit) m = mach_limit;
    return m;
}

// ----------------------------------------------------------------------
// Chang-Cooper face weights: cc_eval_face_weights, Chang_Cooper.c:22-40.
// For |w| >= 0.1 the three exponentials of the reference collapse to one:
// with aw = |w|, -aw/2 + w/2 and -aw/2 - w/2 are exactly 0 and -aw in some
// order, and exp(0) == 1 exactly.
// ----------------------------------------------------------------------
CROMA_HD void face_weights(double w, double &wp, double &wm)
{
    if (fabs(w) < 0.1) {
        const double w2 = w * w;
        const double den = 1.0 + w2 / 24.0 + (w2 * w2) / 1920.0;
        wp = exp(0.5 * w) / den;
        wm = exp(-0.5 * w) / den;
    } else {
        const double aw = fabs(w);
        const double e = exp(-aw);
        const double den = 1.0 - e;
        const double big = aw / den;
        const double small = aw * e / den;
        wp = (w >= 0.0) ? big : small;
        wm = (w >= 0.0) ? small : big;
    }
}

// FP64 reciprocal for the factor and per-step kernels.  CUDA's IEEE division
// is a called routine: on B200 one costs ~125-145 cycles of a warp's time and
// two of them never overlap (measured: the same per-division time at 1, 4 or
// 8 independent divisions per thread), so a chain of pivots or a row of
// faces serialises on it.  This form is inline: the hardware approximation
// (PTX rcp.approx.ftz.f64) and two Newton-Raphson steps for 1/x in FMA form,
// e = 1 - x y, y <- y + y e (each step squares the relative error), which
// reach the FP64 rounding level for normal x (tested against the exact
// reciprocal in ulps).  Subnormal x is flushed (then 0 gives a NaN) and
// 1/x below the normal range returns 0; the callers' operands are O(1)
// denominators bounded away from both.  Host builds divide.
CROMA_HD double rcp_nr(double x)
{
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
#else
    return 1.0 / x;
#endif
}

// FP64 exp for the factor kernels' face weights and Coulomb term: Tang's
// table-driven method (P. T. P. Tang, "Table-driven implementation of the
// exponential function in IEEE floating-point arithmetic", ACM TOMS 15(2),
// 1989).  x = (32 m + j) ln2/32 + r with N = 32 m + j = rint(32 x / ln2)
// (the 1.5 * 2^52 shifter leaves N in the low word), |r| <= ln2/64 by a
// two-part reduction with ln2/32 = kExpLhi + kExpLlo, exp(r) - 1 by its
// Taylor polynomial to degree 6 (truncation below 4e-18), and
// exp(x) = 2^m (2^(j/32) + 2^(j/32) p), the scale applied as two exact
// powers of two so that results down to the subnormal range are formed.
// Within 1 ulp of the exact value in an exact-arithmetic emulation and on
// the device (tested); about half the dependent depth of a general exp,
// which is what the latency-bound factor kernel waits on.  x is clamped to
// [-746, 709] (exp(-746) rounds to 0); a NaN stays a NaN.
static __device__ const double kExp2J[32] = {
    0x1.0000000000000p+0, 0x1.059b0d3158574p+0, 0x1.0b5586cf9890fp+0, 0x1.11301d0125b51p+0,
    0x1.172b83c7d517bp+0, 0x1.1d4873168b9aap+0, 0x1.2387a6e756238p+0, 0x1.29e9df51fdee1p+0,
    0x1.306fe0a31b715p+0, 0x1.371a7373aa9cbp+0, 0x1.3dea64c123422p+0, 0x1.44e086061892dp+0,
    0x1.4bfdad5362a27p+0, 0x1.5342b569d4f82p+0, 0x1.5ab07dd485429p+0, 0x1.6247eb03a5585p+0,
    0x1.6a09e667f3bcdp+0, 0x1.71f75e8ec5f74p+0, 0x1.7a11473eb0187p+0, 0x1.82589994cce13p+0,
    0x1.8ace5422aa0dbp+0, 0x1.93737b0cdc5e5p+0, 0x1.9c49182a3f090p+0, 0x1.a5503b23e255dp+0,
    0x1.ae89f995ad3adp+0, 0x1.b7f76f2fb5e47p+0, 0x1.c199bdd85529cp+0, 0x1.cb720dcef9069p+0,
    0x1.d5818dcfba487p+0, 0x1.dfc97337b9b5fp+0, 0x1.ea4afa2a490dap+0, 0x1.f50765b6e4540p+0};
constexpr double kExpInvL = 0x1.71547652b82fep+5;   // 32 / ln2
constexpr double kExpLhi = 0x1.62e42fefa39efp-6;    // ln2 / 32, leading part
constexpr double kExpLlo = 0x1.abc9e3b39803fp-61;   // ln2 / 32 - kExpLhi

CROMA_HD double exp_tab(double x)
{
#ifdef __CUDA_ARCH__
    x = x < -746.0 ? -746.0 : (x > 709.0 ? 709.0 : x);   // a NaN passes through
    const double t = fma(x, kExpInvL, 0x1.8p52);
    const double n = t - 0x1.8p52;
    const int N = __double2loint(t);
    double r = fma(-n, kExpLhi, x);
    r = fma(-n, kExpLlo, r);
    const double r2 = r * r;
    const double u = fma(1.0 / 6.0, r, 0.5);
    double v = fma(1.0 / 120.0, r, 1.0 / 24.0);
    v = fma(1.0 / 720.0, r2, v);
    const double p = fma(fma(v, r2, u), r2, r);
    const double tj = __ldg(&kExp2J[N & 31]);
    const int m = N >> 5, m1 = m >> 1, m2 = m - m1;
    const double s1 = __hiloint2double((m1 + 1023) << 20, 0), s2 = __hiloint2double((m2 + 1023) << 20, 0);
    return fma(tj, p, tj) * s1 * s2;
#else
    return exp(x);
#endif
}

// The same weights with one exponential and one division per face and no
// divergent branch (the evolve kernels' form): exp(-w/2) is taken as
// 1/exp(w/2), the exponential is exp_tab, the two quotients by the
// denominator share one reciprocal (rcp_nr) and the series constants are
// multiplied in.  Agrees with
// face_weights to a few ulp.
CROMA_HD void face_weights_fast(double w, double &wp, double &wm)
{
    const double aw = fabs(w);
    const bool series = aw < 0.1;
    const double w2 = w * w;
    const double dser = 1.0 + w2 * (1.0 / 24.0) + (w2 * w2) * (1.0 / 1920.0);
    const double e = exp_tab(series ? 0.5 * w : -aw);
    const double q = (series ? 1.0 : aw) * rcp_nr(series ? e * dser : 1.0 - e);
    const double s = q * e;
    // series: wm = 1 / (e dser), wp = e / dser; otherwise big = q, small = q e
    wp = series ? s * e : ((w >= 0.0) ? q : s);
    wm = series ? q : ((w >= 0.0) ? s : q);
}

CROMA_HD double face_delta(double w)
{
    return 1.0 / w - 1.0 / (exp(w) - 1.0);
}

// cc_prepare_face_weight, Chang_Cooper.c:42-64 (delta not produced).
CROMA_HD void face(double bl, double br, double cl, double cr, double xl, double xr,
                   double &wp, double &wm, double &w)
{
    wp = 0.0; wm = 0.0; w = 0.0;
    if (fabs(cl) <= 1.0e-200) return;
    w = 0.5 * (bl + br) / (0.5 * (cl + cr)) * (xr - xl);
    face_weights(w, wp, wm);
}

// ----------------------------------------------------------------------
// Inverse-Compton cooling (FP_Coef.c:361-436, 480-539)
// ----------------------------------------------------------------------
struct IcConsts {
    double cmb_pref;      // 8 pi c c c pow(m_e/h, 3) (FP_Coef.c:402)
    double cmb_pref_d;    // same with the derivative's constants (FP_Coef.c:412)
    double k_d;           // 1.38 * pow(10, -16) (FP_Coef.c:410)
    double log10_90;      // 90 log(10)
};

CROMA_HD double ic_kernel(double eps0, double gamma, double eps)   // IC_kernel :379-389
{
    const double re = 2.82e-13;
    const double kappa = eps / (4.0 * eps0 * gamma * (gamma - eps));
    if (kappa <= 0.0) return 0.0;
    const double t = 4.0 * eps0 * kappa * gamma;
    double C = 2.0 * kappa * log(kappa) + (1.0 + 2.0 * kappa) * (1.0 - kappa) +
               (t * t) / (2.0 * (1.0 + 4.0 * eps0 * gamma * kappa)) * (1.0 - kappa);
    return 2.0 * kPi * re * re * kC / (gamma * gamma * eps0) * C;
}

CROMA_HD double cmb_density(const IcConsts &k, double eps, double z)   // :391-406
{
    const double Tcmb = 2.757 * (1.0 + z);
    const double X = eps * 9.11e-28 * kC * kC / (1.38e-16 * Tcmb);
    if (X > k.log10_90) return 0.0;
    const double ex = exp(X);
    if (ex - 1.0 < 1.0e-40) {
        return k.cmb_pref * eps / (9.11e-28 * kC * kC * (1.0 + 0.5 * X + X / 6.0) / (1.38e-16 * Tcmb));
    }
    return k.cmb_pref * (eps * eps) / (ex - 1.0);
}

CROMA_HD double cmb_density_deps(const IcConsts &k, double eps, double z)   // :407-413
{
    const double Tcmb = 2.757 * (1.0 + z);
    const double X = eps * 9.11e-28 * kC * kC / (k.k_d * Tcmb);
    const double ex = exp(X);
    return k.cmb_pref_d * eps / (ex - 1.0) *
           (2.0 - eps * 9.11e-28 * kC * kC * ex / (k.k_d * Tcmb * (ex - 1.0)));
}

// Inner integral b_IC_integrand (FP_Coef.c:512-539)
CROMA_HD double b_ic_integrand(double eps0, double gamma, double emin, double emax)
{
    const double da = 0.50e-1;
    const int N = (int)round((log10(emax) - log10(emin)) / da);
    double a = log10(emin), epsnew = emin, integral = 0.0;
    double newC = ic_kernel(eps0, gamma, epsnew);
    for (int i = 0; i < N; i++) {
        a = a + da;
        const double eps = epsnew;
        epsnew = pow(10.0, a);
        const double deps = epsnew - eps;
        const double C = newC;
        newC = ic_kernel(eps0, gamma, epsnew);
        integral = integral + 0.5 * (eps * C + epsnew * newC) * deps;
    }
    return integral;
}

// IC_emissivity_kernel, FP_Coef.c:553-584: the inverse-Compton emissivity of
// one electron of Lorentz factor gamma at frequency nu (Hz), a 400-step
// log-spaced trapezoid over the seed CMB photon energy.  The photon energy
// is normalised with the routine's own c = 3.0e10.
CROMA_HD double ic_emissivity(const IcConsts &k, double nu, double gamma, double z)
{
    const int N = 400;
    const double meg = 9.11e-28, c_local = 3.0e+10;
    const double eps = kHPlanck * nu / (meg * c_local * c_local);
    const double e0max = eps;
    double e0min = eps / (4.0 * gamma * (gamma - eps));
    if (e0min < 0) e0min = eps / (gamma * gamma);
    const double da = (log10(e0max) - log10(e0min)) / (double)N;
    double a = log10(e0min);
    double eps0new = pow(10.0, a);
    double Cnew = ic_kernel(eps0new, gamma, eps);
    double n0new = cmb_density(k, eps0new, z);
    double integral = 0.0;
    for (int i = 0; i < N; i++) {
        a = a + da;
        const double eps0 = eps0new;
        eps0new = pow(10.0, a);
        const double deps0 = eps0new - eps0;
        const double C = Cnew, n = n0new;
        n0new = cmb_density(k, eps0new, z);
        Cnew = ic_kernel(eps0new, gamma, eps);
        integral = integral + 0.5 * (C * n + Cnew * n0new) * deps0;
    }
    return kHPlanck * eps * integral / (4.0 * kPi);
}

}  // namespace croma
