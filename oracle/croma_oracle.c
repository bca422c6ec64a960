/*
 * croma_oracle.c -- CPU restatement of CROMA's per-tracer Fokker-Planck
 * update.  TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker.
 * The product (libcroma_b200_np*.so) neither links nor calls it.
 *
 * Every routine names the reference file:line whose algorithm it restates
 * (paths relative to the kosukenishiwaki/croma-fp tree).  Arithmetic is kept
 * in the reference's evaluation order so that, compiled with the same libm,
 * the restatement reproduces the reference's own CPU results; the test
 * suite pins it against oracle/_ref (the reference sources compiled as-is).
 */
#include "croma_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Physical constants: src/CONSTANTS.c:3-19. */
static const double K_C = 2.999e+10;
static const double K_GEV = 1.6e-3;
static const double K_EV = 1.6e-12;
static const double K_MSUN = 1.99e+33;
static const double K_MPC = 3.0857e+24;
static const double K_KPC = 3.0857e+21;
static const double K_GYR = 3.1536e+16;
static const double K_HPLANCK = 6.63e-27;
static const double K_MP = 0.938;
static const double K_ME = 0.511e-3;
static const double K_MB = 1.0e-27;
static const double K_MPI_CH = 1.40e-1;
static const double K_MMU = 1.05e-1;

typedef struct {
    double *p, *dp, *E;
    double pm1, pp1;
} OrGrid;

struct OrCtx {
    OrParams par;
    int nb;
    OrGrid crp, cre;
    double *beta_p;
    /* grid cache: src/FP_Coef.c:27-156 */
    double *crp_p2, *crp_exp_cut, *crp_sigma_pp, *crp_sigmoid_pp;
    int crp_j_pp;
    double crp_pm1_p2, crp_pp1_p2, crp_pm1_exp_cut, crp_pp1_exp_cut;
    double *cre_p2, *cre_exp_cut;
    double cre_pm1_p2, cre_pp1_p2, cre_pm1_exp_cut, cre_pp1_exp_cut;
    /* secondary-electron weights, transposed [jp][je]: src/fp_shared_core.c:1453-1506 */
    double *fqe;
    int *np_min_qe;
    int fqe_jp0;
};

/* ------------------------------------------------------------------ */
/* Momentum grid: momentum_bin, src/FP_Coef.c:291-330                  */
/* ------------------------------------------------------------------ */
static void or_build_grid(OrCtx *ctx)
{
    const int n = ctx->nb;
    double a, da;
    int j;

    da = (ctx->par.pmax - ctx->par.pmin) / (double)n;
    a = ctx->par.pmin - da;
    ctx->crp.pm1 = pow(10.0, a);
    for (j = 0; j < n; j++) {
        a = a + da;
        ctx->crp.p[j] = pow(10.0, a);
        ctx->crp.E[j] = K_MP * sqrt(1.0 + ctx->crp.p[j] * ctx->crp.p[j]);
        ctx->beta_p[j] = ctx->crp.p[j] / sqrt(1.0 + ctx->crp.p[j] * ctx->crp.p[j]);
    }
    a = a + da;
    ctx->crp.pp1 = pow(10.0, a);
    for (j = 1; j < n - 1; j++) ctx->crp.dp[j] = 0.5 * (ctx->crp.p[j + 1] - ctx->crp.p[j - 1]);
    ctx->crp.dp[0] = 0.5 * (ctx->crp.p[1] - ctx->crp.pm1);
    ctx->crp.dp[n - 1] = 0.5 * (pow(10.0, a + da) - ctx->crp.p[n - 2]);

    da = (ctx->par.pemax - ctx->par.pemin) / (double)n;
    a = ctx->par.pemin - da;
    ctx->cre.pm1 = pow(10.0, a);
    for (j = 0; j < n; j++) {
        a += da;
        ctx->cre.p[j] = pow(10.0, a);
        ctx->cre.E[j] = K_ME * sqrt(1.0 + ctx->cre.p[j] * ctx->cre.p[j]);
    }
    a += da;
    ctx->cre.pp1 = pow(10.0, a);
    for (j = 1; j < n - 1; j++) ctx->cre.dp[j] = 0.5 * (ctx->cre.p[j + 1] - ctx->cre.p[j - 1]);
    ctx->cre.dp[0] = 0.5 * (ctx->cre.p[1] - ctx->cre.pm1);
    ctx->cre.dp[n - 1] = 0.5 * (pow(10.0, a + da) - ctx->cre.p[n - 2]);
}

/* ------------------------------------------------------------------ */
/* Kamae (2006) pion cross section: pp_pion_cross_section,            */
/* src/HADRONIC.c:342-429                                              */
/* ------------------------------------------------------------------ */
static double or_pp_pion_xsec(int kind, double p)
{
    static const double a0 = 0.1176, a1 = 0.3829, a2 = 23.10, a3 = 6.454, a4 = -5.764,
                        a5 = -23.63, a6 = 94.75, a7 = 0.02667;
    static const double b0 = 11.34, b1 = 23.72;
    static const double c0 = 28.5, c1 = -6.133, c2 = 1.464;
    static const double d0 = 0.3522, d1 = 0.1530, d2 = 1.498, d3 = 2.0, d4 = 30.0,
                        d5 = 3.155, d6 = 1.042;
    static const double e0 = 5.922, e1 = 1.632;
    static const double f0 = 0.0834, f1 = 9.5, f2 = 5.5, f3 = 1.68, f4 = 3134.0;
    static const double g0 = 0.0004257, g1 = 4.5, g2 = 7.0, g3 = 2.1, g4 = 503.5;
    double Ep, Tp, x, x2, x3, nondiff, diff, dres, res, tot, r0, rp, rm;

    if (kind > 2 || kind < -2) return 0.0;
    Ep = sqrt(K_MP * K_MP + p * p);
    Tp = Ep - K_MP;
    x = log10(p);
    x2 = x * x;
    x3 = x2 * x;

    if (p < 1.0) nondiff = 0.0;
    else if (p < 1.3) nondiff = 0.57 * pow(x / a0, 1.2) * (a2 + a3 * x2 + a4 * x3 + a5 * exp(-a6 * pow(x + a7, 2.0)));
    else if (p < 2.4) nondiff = (b0 * fabs(a1 - x) + b1 * fabs(a0 - x)) / (a1 - a0);
    else if (p < 10.0) nondiff = a2 + a3 * x2 + a4 * x3 + a5 * exp(-a6 * pow(x + a7, 2.0));
    else nondiff = c0 + c1 * x + c2 * x2;

    if (p < 2.25) diff = 0.0;
    else if (p < 3.2) diff = sqrt(fabs(x - d0) / d1) * (d2 + d3 * log10(d4 * (x - 0.25)) + d5 * x2 - d6 * x3);
    else if (p < 100.0) diff = d2 + d3 * log10(d4 * (x - 0.25)) + d5 * x2 - d6 * x3;
    else diff = e0 + e1 * x;

    if (Ep < 1.4) dres = 0.0;
    else if (Ep < 1.6) dres = f0 * pow(Ep, 10.0);
    else if (Ep < 1.8) dres = f1 * exp(-f2 * pow(Ep - f3, 2.0));
    else if (Ep < 10.0) dres = f4 * pow(Ep, -10.0);
    else dres = 0.0;

    if (Ep < 1.6) res = 0.0;
    else if (Ep < 1.9) res = g0 * pow(Ep, 14.0);
    else if (Ep < 2.3) res = g1 * exp(-g2 * pow(Ep - g3, 2.0));
    else if (Ep < 20.0) res = g4 * pow(Ep, -6.0);
    else res = 0.0;

    tot = (nondiff + diff + dres + res) * K_MB;
    /* Blattnig (2000) charge scaling */
    r0 = 1.0 / (0.007 + 0.1 * log(Tp) / Tp + 0.3 / Tp / Tp);
    rp = 1.0 / (0.00717 + 0.0652 * log(Tp) / Tp + 0.162 / Tp / Tp);
    rm = 1.0 / (0.00456 + 0.0846 / pow(Tp, 0.5) + 0.577 / pow(Tp, 1.5));
    if (kind == 0) return tot;
    if (kind == 1) return tot * rp / r0;
    if (kind == -1) return tot * rm / r0;
    return tot * (1.0 + rp / r0 + rm / r0);
}

/* Grid caches: src/FP_Coef.c:77-156 (p_cut = pe_cut = 1). */
static void or_build_grid_cache(OrCtx *ctx)
{
    const int n = ctx->nb;
    const double p_cut = 1.0;
    int j, j_pp = 0;
    double p_pp;

    for (j = 0; j < n; j++) {
        ctx->crp_p2[j] = ctx->crp.p[j] * ctx->crp.p[j];
        ctx->crp_exp_cut[j] = exp(-p_cut / ctx->crp.p[j]);
        ctx->crp_sigma_pp[j] = or_pp_pion_xsec(2, K_MP * ctx->crp.p[j]);
    }
    for (j = 0; j < n - 100; j++) {
        if (j_pp == 0 && ctx->crp_sigma_pp[j] > 0.0) j_pp = j;
    }
    j_pp += 2;
    if (j_pp < 0) j_pp = 0;
    if (j_pp >= n) j_pp = n - 1;
    ctx->crp_j_pp = j_pp;
    p_pp = ctx->crp.p[j_pp];
    for (j = 0; j < n; j++)
        ctx->crp_sigmoid_pp[j] = 1.0 / (1.0 + exp(-5.0 * (ctx->crp.p[j] - p_pp)));
    ctx->crp_pm1_p2 = ctx->crp.pm1 * ctx->crp.pm1;
    ctx->crp_pp1_p2 = ctx->crp.pp1 * ctx->crp.pp1;
    ctx->crp_pm1_exp_cut = exp(-p_cut / ctx->crp.pm1);
    ctx->crp_pp1_exp_cut = exp(-p_cut / ctx->crp.pp1);

    for (j = 0; j < n; j++) {
        ctx->cre_p2[j] = ctx->cre.p[j] * ctx->cre.p[j];
        ctx->cre_exp_cut[j] = exp(-p_cut / ctx->cre.p[j]);
    }
    ctx->cre_pm1_p2 = ctx->cre.pm1 * ctx->cre.pm1;
    ctx->cre_pp1_p2 = ctx->cre.pp1 * ctx->cre.pp1;
    ctx->cre_pm1_exp_cut = exp(-p_cut / ctx->cre.pm1);
    ctx->cre_pp1_exp_cut = exp(-p_cut / ctx->cre.pp1);
}

/* ------------------------------------------------------------------ */
/* Secondary electrons: QeKernel_BB05 and helpers,                     */
/* src/HADRONIC.c:291-335, 431-533                                     */
/* ------------------------------------------------------------------ */
static double or_fpiq(int m, double Epi, double Ep)   /* FpiQ, HADRONIC.c:324-336 */
{
    double L = log(0.001 * Ep), x = Epi / Ep, mpi = 1.35e-1;
    double Bpi, alpha, r, xa, A;
    if (m == 1) mpi = 1.40e-1;
    if (m == 0) mpi = 1.35e-1;
    if (x <= mpi / Ep) return 0.0;
    if (x > 1.0) return 0.0;
    Bpi = 5.58 + 0.78 * L + 0.10 * L * L;
    alpha = 0.89 / (sqrt(Bpi) * (1.0 - exp(-0.33 * Bpi)));
    r = 3.1 / (pow(Bpi, 1.5));
    xa = pow(x, alpha);
    A = pow((1.0 - xa) / pow(1.0 + r * xa, 3.0), 4.0);
    A = A * (1.0 / (1.0 - xa) + 3.0 * r / (1.0 + r * xa)) * sqrt(1.0 - mpi / (x * Ep));
    return 4.0 * alpha * Bpi * xa * A / x / Ep;
}

static double or_dsigma(int i, double Epi, double Ep)  /* dsigma, HADRONIC.c:291-300 */
{
    double gp = Ep / K_MP, gbp = sqrt(gp * gp - 1.0), pp = gbp * K_MP;
    double Fpi = or_fpiq(0, Epi, Ep);
    double s = or_pp_pion_xsec(i, pp);
    return s * Fpi / sqrt(1.0 + 1.0 / (gbp * gbp));
}

static double or_lorentz_beta(double gamma)            /* HADRONIC.c:431-435 */
{
    double b2 = gamma * gamma - 1.0;
    if (b2 < 0.0) return 0.0;
    return sqrt(b2) / gamma;
}

static double or_fe_bl10(double Ee, double Epi)        /* Fe, HADRONIC.c:499-533 */
{
    const double mpi = 1.3957e-1, mmu = 1.05658e-1, bmu = 0.2714;
    double gpi = Epi / mpi;
    double xi = mmu * mmu / (mpi * mpi);
    double Emu = (mpi * mpi - mmu * mmu) / (mpi * mpi) * Epi / (2.0 * bmu);
    double betamu = sqrt(1.0 - mmu * mmu / (Emu * Emu));
    double lambda = 2.0 * mpi * mpi * Ee * bmu / ((mpi * mpi - mmu * mmu) * Epi);
    double P, X, l2 = lambda * lambda, l3 = l2 * lambda;
    P = 1.0 / betamu * (2.0 * Epi * xi / (Emu * (1.0 - xi)) - (1.0 + xi) / (1.0 - xi));
    if (lambda > 1.0) return 0.0;
    if (gpi == 1.0) return 0.0;
    if (lambda < 0.0) return 0.0;
    if ((1.0 - betamu) / (1.0 + betamu) < lambda) {
        X = 5.0 - 9.0 * l2 + 4.0 * l3 -
            P / betamu * (1.0 - (6.0 * betamu + 3.0) * l2 + (6.0 * betamu + 2.0) * l3);
        return X / 12.0;
    } else if (lambda < (1.0 - betamu) / (1.0 + betamu)) {
        X = l2 * betamu / pow(1.0 - betamu, 2.0) *
                (3.0 - 2.0 / 3.0 * lambda * (3.0 + betamu * betamu) / (1.0 - betamu)) -
            P / (1.0 - betamu) *
                (l2 * (1.0 + betamu) - 2.0 * l2 / (1.0 - betamu) * (0.5 + lambda * (1.0 + betamu)) +
                 2.0 * l3 * (3.0 + betamu * betamu) / (3.0 * pow(1.0 - betamu, 2.0)));
        return X;
    }
    return 0.0;
}

static double or_qe_kernel(double Ee, double p)        /* QeKernel_BB05, HADRONIC.c:436-497 */
{
    const double bmu = 0.2714;
    double gp = sqrt(p * p + 1.0), Ep = gp * K_MP, Emax = gp * K_MP;
    double r = 0.5 * (K_MPI_CH * K_MPI_CH - K_MMU * K_MMU) / (bmu * K_MPI_CH * K_MPI_CH);
    double Emin = Ee / r, amin, amax, a, Epi, Emu, betamu, f, fpre, Epipre, dEpi, integral = 0.0;
    const double da = 0.05;
    int Na, i;

    if (Emax < Emin || (Ep - K_MP) < 0.289) return 0;
    Emin = fmax(Emin, K_MPI_CH);
    amin = log10(Emin);
    amax = log10(Emax);
    Na = (int)fmax(50, round((amax - amin) / da));
    a = amin;
    Epi = pow(10.0, a);
    Emu = Epi * r;
    betamu = or_lorentz_beta(Emu / K_MMU);
    if (betamu == 0.0) f = 0.0;
    else f = (or_dsigma(1, Epi, Ep) + or_dsigma(-1, Epi, Ep)) * or_fe_bl10(Ee, Epi) / (betamu * Epi);
    for (i = 1; i < Na; i++) {
        Epipre = Epi;
        a = a + da;
        Epi = pow(10.0, a);
        dEpi = Epi - Epipre;
        fpre = f;
        Emu = Epi * r;
        betamu = or_lorentz_beta(Emu / K_MMU);
        f = (or_dsigma(1, Epi, Ep) + or_dsigma(-1, Epi, Ep)) * or_fe_bl10(Ee, Epi) / (betamu * Epi);
        integral = integral + 0.5 * (f + fpre) * dEpi;
        if (integral < 0.0 || isnan(integral)) return 0.0;
    }
    return 8.0 * bmu * K_MPI_CH * K_MPI_CH * (K_C * K_ME) * integral /
           (K_MPI_CH * K_MPI_CH - K_MMU * K_MMU);
}

/* prepare_secondary_kernel_flat, src/fp_shared_core.c:1453-1506
 * (transposed layout, the reference default). */
static void or_build_secondary_kernel(OrCtx *ctx)
{
    const int n = ctx->nb;
    double *vals = (double *)malloc((size_t)n * sizeof(double));
    int je, jp;

    for (je = 0; je < n; je++) {
        int jp0;
        for (jp = 0; jp < n; jp++) {
            double v = or_qe_kernel(ctx->cre.E[je], ctx->crp.p[jp]) * ctx->beta_p[jp];
            if (isnan(v)) v = 0.0;
            vals[jp] = v;
        }
        ctx->np_min_qe[je] = 1;
        for (jp = 1; jp < n; jp++)
            if (vals[jp] < 1.0e-80) ctx->np_min_qe[je] = jp;
        jp0 = ctx->np_min_qe[je];
        if (jp0 < 1) jp0 = 1;
        if (jp0 > n) jp0 = n;
        for (jp = 0; jp < n; jp++) {
            double w = 0.0;
            if (jp0 < n) {
                if (jp == jp0 - 1) w = 0.5 * vals[jp] * ctx->crp.dp[jp0];
                else if (jp >= jp0 && jp < n - 1) w = 0.5 * vals[jp] * (ctx->crp.dp[jp] + ctx->crp.dp[jp + 1]);
                else if (jp == n - 1 && jp >= jp0) w = 0.5 * vals[jp] * ctx->crp.dp[jp];
            }
            ctx->fqe[(size_t)jp * n + je] = w;
        }
        ctx->np_min_qe[je] = (jp0 < n) ? (jp0 - 1) : n;
    }
    /* first proton bin that any electron bin draws from:
     * src/fp_shared_core.c:1615-1623 */
    ctx->fqe_jp0 = n;
    for (je = 0; je < n; je++) {
        int j0 = ctx->np_min_qe[je];
        if (j0 < 0) j0 = 0;
        if (j0 < ctx->fqe_jp0) ctx->fqe_jp0 = j0;
    }
    free(vals);
}

/* ------------------------------------------------------------------ */
/* Inverse-Compton cooling row: rad_IC_cool and helpers,               */
/* src/FP_Coef.c:361-436, 485-539                                      */
/* ------------------------------------------------------------------ */
static double or_ic_kernel(double eps0, double gamma, double eps)   /* IC_kernel :379-389 */
{
    const double re = 2.82e-13;
    double kappa = eps / (4.0 * eps0 * gamma * (gamma - eps)), C;
    if (kappa <= 0.0) return 0.0;
    C = 2.0 * kappa * log(kappa) + (1.0 + 2.0 * kappa) * (1.0 - kappa) +
        pow(4.0 * eps0 * kappa * gamma, 2.0) / (2.0 * (1.0 + 4.0 * eps0 * gamma * kappa)) * (1.0 - kappa);
    return 2.0 * M_PI * re * re * K_C / (gamma * gamma * eps0) * C;
}

static double or_cmb_density(double eps, double z)                  /* :391-406 */
{
    const double T0 = 2.757, meg = 9.11e-28, k = 1.38e-16, epsilon = 1.0e-40;
    double Tcmb = T0 * (1.0 + z), x;
    if (eps * meg * K_C * K_C / (k * Tcmb) > 90.0 * log(10.0)) return 0;
    if (exp(eps * meg * K_C * K_C / (k * Tcmb)) - 1.0 < epsilon) {
        x = eps * meg * K_C * K_C / (k * Tcmb);
        return 8.0 * M_PI * K_C * K_C * K_C * pow(meg / K_HPLANCK, 3.0) * eps /
               (meg * K_C * K_C * (1.0 + 0.5 * x + x / 6.0) / (k * Tcmb));
    }
    return 8.0 * M_PI * K_C * K_C * K_C * pow(meg / K_HPLANCK, 3.0) * pow(eps, 2.0) /
           (exp(eps * meg * K_C * K_C / (k * Tcmb)) - 1.0);
}

static double or_cmb_density_deps(double eps, double z)             /* :407-413 */
{
    const double h = 6.63e-27, T0 = 2.757, meg = 9.11e-28;
    const double k = 1.38 * pow(10.0, -16.0);
    double Tcmb = T0 * (1.0 + z);
    return 8.0 * M_PI * K_C * K_C * K_C * pow(meg / h, 3.0) * eps /
           (exp(eps * meg * K_C * K_C / (k * Tcmb)) - 1.0) *
           (2.0 - eps * meg * K_C * K_C * exp(eps * meg * K_C * K_C / (k * Tcmb)) /
                      (k * Tcmb * (exp(eps * meg * K_C * K_C / (k * Tcmb)) - 1.0)));
}

static void or_cmb_bounds(double z, double *emin, double *emax)     /* :414-436 */
{
    const double delta = pow(10.0, -5.5);
    const double meg = 9.11 * pow(10.0, -28.0), cl = 3.0e+10, T0 = 2.725;
    const double k = 1.38 * pow(10.0, -16.0);
    double epsp = k / (meg * cl * cl) * T0 * (1.0 + z);
    double peak = or_cmb_density(epsp, z);
    double eps, epsnew;
    int it;

    epsnew = 0.01 * epsp;
    eps = 1.0;
    for (it = 0; fabs(epsnew - eps) > delta * eps && it < 100000; it++) {
        eps = epsnew;
        epsnew = eps - (or_cmb_density(eps, z) - peak * delta) / or_cmb_density_deps(eps, z);
    }
    *emin = epsnew;
    epsnew = 10.0 * epsp;
    eps = 1.0;
    for (it = 0; fabs(epsnew - eps) > delta * eps && it < 100000; it++) {
        eps = epsnew;
        epsnew = eps - (or_cmb_density(eps, z) - peak * delta) / or_cmb_density_deps(eps, z);
    }
    *emax = epsnew;
}

static double or_b_ic_integrand(double eps0, double gamma, double emin, double emax) /* :512-539 */
{
    const double da = 0.50e-1;
    int i, N = (int)round((log10(emax) - log10(emin)) / da);
    double a = log10(emin), eps, epsnew = emin, deps, C, newC, integral = 0.0;
    newC = or_ic_kernel(eps0, gamma, epsnew);
    for (i = 0; i < N; i++) {
        a = a + da;
        eps = epsnew;
        epsnew = pow(10.0, a);
        deps = epsnew - eps;
        C = newC;
        newC = or_ic_kernel(eps0, gamma, epsnew);
        integral = integral + 0.5 * (eps * C + epsnew * newC) * deps;
    }
    return integral;
}

static double or_b_ic(double gamma, double e0min, double e0max, double z)   /* :480-511 */
{
    const double da = 0.50e-1;
    int i, N = (int)round((log10(e0max) - log10(e0min)) / da);
    double a = log10(e0min), e0, e0new = e0min, emin, emax, n, n0new, IC2, IC2new, deps0;
    double integral = 0.0;
    emin = e0new;
    emax = gamma * 4.0 * e0new * gamma / (1.0 + 4.0 * e0new * gamma);
    IC2new = or_b_ic_integrand(e0new, gamma, emin, emax);
    n0new = or_cmb_density(e0new, z);
    for (i = 0; i < N; i++) {
        a = a + da;
        e0 = e0new;
        n = n0new;
        IC2 = IC2new;
        e0new = pow(10.0, a);
        n0new = or_cmb_density(e0new, z);
        deps0 = e0new - e0;
        emin = e0new;
        emax = gamma * 4.0 * e0new * gamma / (1.0 + 4.0 * e0new * gamma);
        IC2new = or_b_ic_integrand(e0new, gamma, emin, emax);
        integral = integral + 0.5 * (n * IC2 + n0new * IC2new) * deps0;
    }
    return integral * K_GYR;
}

int or_ic_row(const OrCtx *ctx, double z, double *row, double *m1, double *p1)
{
    double e0min, e0max;
    int j;
    if (ctx == 0 || row == 0 || m1 == 0 || p1 == 0) return -1;
    or_cmb_bounds(z, &e0min, &e0max);
    for (j = 0; j < ctx->nb; j++)
        row[j] = or_b_ic(sqrt(1.0 + ctx->cre.p[j] * ctx->cre.p[j]), e0min, e0max, z);
    *m1 = or_b_ic(sqrt(1.0 + ctx->cre.pm1 * ctx->cre.pm1), e0min, e0max, z);
    *p1 = or_b_ic(sqrt(1.0 + ctx->cre.pp1 * ctx->cre.pp1), e0min, e0max, z);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Loss rates                                                          */
/* ------------------------------------------------------------------ */
static double or_coulomb_kernel(double x)          /* b_Coulomb_kernel, FP_Coef.c:451-453 */
{
    return 0.5 * sqrt(M_PI) * erf(sqrt(x)) - sqrt(x) * exp(-x);
}

static double or_b_coulomb_p(double n, double p, double kbt)   /* b_Coulomb_p, FP_Coef.c:438-449 */
{
    const double p2 = p * p;
    const double gamma = sqrt(1.0 + p2);
    const double betap2 = p2 / (1.0 + p2);
    const double kinetic = gamma - 1.0;
    const double Ep = gamma * K_MP - K_MP;
    double xp = Ep / kbt, xe = xp * (K_ME / K_MP);
    double sum = or_coulomb_kernel(xe) + or_coulomb_kernel(xp) * (K_ME / K_MP);
    double thermal = 1.0 - kbt / (2.0 * K_MP * kinetic);
    if (thermal < 0.0) return 0.0;
    return K_GYR * K_C / (K_MP * K_GEV) * sum * n * (1.0 / betap2) * thermal * 3.5e-29;
}

static double or_b_synch(double p, double B)       /* b_synch, FP_Coef.c:454-462 */
{
    const double b_ratio = B * 1.0e+6 / 3.2;
    return 4.8e-4 * p * p * b_ratio * b_ratio * 9.11e-28 * 3.0e+10 * 3.1536e+16;
}

static double or_b_coulomb_e(double n, double pe)  /* b_Coulomb_e, FP_Coef.c:464-469 */
{
    const double pe2 = pe * pe;
    double beta2 = pe2 / (1.0 + pe2);
    return 3.05e-29 * n * (1.0 + log(pe / n) / 74.8) / (K_ME * K_GEV) * K_C * K_GYR / beta2;
}

/* prepare_crp_losses_1d_with_threshold, src/fp_shared_core.c:729-778 */
static void or_crp_losses(const OrCtx *ctx, double n_gas, double kbt, double divv,
                          double *radp, double *tloss, double *radpm1, double *radpp1)
{
    const double kappa_pp = 0.5;
    const double tloss_pref = 1.0 / (kappa_pp * K_C * n_gas) / K_GYR;
    const double adiab = 1.0 / 3.0 * divv;
    int j;
    for (j = 0; j < ctx->nb; j++) {
        const double p = ctx->crp.p[j];
        double sig = (j > ctx->crp_j_pp) ? ctx->crp_sigma_pp[j] : ctx->crp_sigma_pp[ctx->crp_j_pp];
        sig *= ctx->crp_sigmoid_pp[j];
        radp[j] = or_b_coulomb_p(n_gas, p, kbt) + adiab * p;
        tloss[j] = tloss_pref / sig;
    }
    *radpm1 = or_b_coulomb_p(n_gas, ctx->crp.pm1, kbt);
    *radpp1 = or_b_coulomb_p(n_gas, ctx->crp.pp1, kbt);
}

/* prepare_cre_losses_1d, src/fp_shared_core.c:780-842 */
static void or_cre_losses(const OrCtx *ctx, double n_gas, double b_field, double divv,
                          const double *rad_ic, double rad_ic_m1, double rad_ic_p1,
                          double *radp, double *tloss, double *radpm1, double *radpp1)
{
    const double b_ratio = b_field * 1.0e+6 / 3.2;
    const double synch_coeff = 4.8e-4 * b_ratio * b_ratio * 9.11e-28 * 3.0e+10 * 3.1536e+16;
    const double coulomb_coeff = 3.05e-29 * n_gas * K_C * K_GYR / (K_ME * K_GEV);
    const double adiab = 1.0 / 3.0 * divv;
    int j;
    for (j = 0; j < ctx->nb; j++) {
        const double pe = ctx->cre.p[j];
        const double pe2 = ctx->cre_p2[j];
        const double beta2 = pe2 / (1.0 + pe2);
        const double coulomb = coulomb_coeff * (1.0 + log(pe / n_gas) / 74.8) / beta2;
        radp[j] = synch_coeff * pe2 + rad_ic[j] + coulomb + adiab * pe;
        tloss[j] = 1.0e+100;
    }
    {
        const double b2m = ctx->cre_pm1_p2 / (1.0 + ctx->cre_pm1_p2);
        const double b2p = ctx->cre_pp1_p2 / (1.0 + ctx->cre_pp1_p2);
        const double cm = coulomb_coeff * (1.0 + log(ctx->cre.pm1 / n_gas) / 74.8) / b2m;
        const double cp = coulomb_coeff * (1.0 + log(ctx->cre.pp1 / n_gas) / 74.8) / b2p;
        *radpm1 = synch_coeff * ctx->cre_pm1_p2 + rad_ic_m1 + cm;
        *radpp1 = synch_coeff * ctx->cre_pp1_p2 + rad_ic_p1 + cp;
    }
}

/* ------------------------------------------------------------------ */
/* Momentum diffusion                                                  */
/* ------------------------------------------------------------------ */
static double or_i_theta(double x)                 /* I_theta, FP_Coef.c:624-626 */
{
    return pow(x, 4.0) / 4.0 + pow(x, 2.0) - (1.0 + 2.0 * x * x) * log(x) - 5.0 / 4.0;
}

static double or_tacc_ttd(const OrCtx *ctx, double L, double cs, double Ms, double v)
{                                                  /* accelerationtime_TTD, FP_Coef.c:629-661 */
    const double x = cs / K_C;
    if (ctx->par.ttd_tacc_model == 1) {
        const double t_norm = 2.5e-3, l_norm = 300.0 * K_KPC, cs_norm = 1500.0e5;
        const double theta = or_i_theta(x);
        if (!(x > 0.0) || !(theta > 0.0) || !(Ms > 0.0) || !(L > 0.0) || !(cs > 0.0)) return 0.0;
        return t_norm / (x * theta) * pow(Ms / 0.5, -4.0) * (L / l_norm) * pow(cs / cs_norm, -1.0);
    } else {
        double kL = 2.0 * M_PI / L;
        double k_cut = 1.04e+4 * pow(Ms, 4.0) * kL;
        double kWk_L = 0.5 * pow(v, 2.0);
        double kWk_cut = kWk_L * pow(k_cut / kL, -0.5);
        return K_C / M_PI / or_i_theta(x) / k_cut / kWk_cut / K_GYR;
    }
}

static double or_tacc_asa(const OrCtx *ctx, double L, double cs, double Ms, double beta_pl)
{                                                  /* accelerationtime_ASA, FP_Coef.c:663-666 */
    return sqrt(6.0 / 5.0) / 12.0 * (K_C / cs / cs) * L / sqrt(beta_pl) / pow(Ms, 3.0) *
           pow(ctx->par.psi, 3.0) / K_GYR;
}

static double or_effective_mach(const OrCtx *ctx, double dv, double cs)  /* FP_Coef.c:668-678 */
{
    double mach;
    if (cs <= 0.0) return 0.0;
    mach = dv / cs;
    if (mach < 0.0) mach = 0.0;
    if (ctx->par.mach_limit > 0.0 && mach > ctx->par.mach_limit) mach = ctx->par.mach_limit;
    return mach;
}

typedef struct {
    double *dpp, *dppe;     /* [nb] each */
    double m1, p1, em1, ep1;
} OrDpp;

static void or_dpp_off(const OrCtx *ctx, OrDpp *d)  /* momentumdiff_off, FP_Coef.c:826-849 */
{
    const double inv = 1.0 / (4.0 * 1.0e+5);
    int j;
    for (j = 0; j < ctx->nb; j++) d->dpp[j] = ctx->crp_p2[j] * inv;
    d->p1 = ctx->crp_pp1_p2 * inv;
    d->m1 = ctx->crp_pm1_p2 * inv;
    for (j = 0; j < ctx->nb; j++) d->dppe[j] = ctx->cre_p2[j] * inv;
    d->ep1 = ctx->cre_pp1_p2 * inv;
    d->em1 = ctx->cre_pm1_p2 * inv;
}

/* momentumdiff_fill_from_tacc (FP_Coef.c:680-716, inv = 1/((q+2) t_acc))
 * and momentumdiff_fill_direct_tacc (:718-754, inv = 1/(4 t_acc)) */
static void or_dpp_fill(const OrCtx *ctx, double inv, double epmax, OrDpp *d)
{
    int j;
    for (j = 0; j < ctx->nb; j++)
        d->dpp[j] = ctx->crp_p2[j] * inv * exp(-ctx->crp.E[j] / epmax) * ctx->crp_exp_cut[j];
    d->p1 = ctx->crp_pp1_p2 * inv * exp(-K_MP * sqrt(1.0 + ctx->crp.pp1 * ctx->crp.pp1) / epmax) *
            ctx->crp_pp1_exp_cut;
    d->m1 = ctx->crp_pm1_p2 * inv * exp(-K_MP * sqrt(1.0 + ctx->crp.pm1 * ctx->crp.pm1) / epmax) *
            ctx->crp_pm1_exp_cut;
    for (j = 0; j < ctx->nb; j++) d->dppe[j] = ctx->cre_p2[j] * inv * ctx->cre_exp_cut[j];
    d->ep1 = ctx->cre_pp1_p2 * inv * ctx->cre_pp1_exp_cut;
    d->em1 = ctx->cre_pm1_p2 * inv * ctx->cre_pm1_exp_cut;
}

/* fp_momentumdiff_tacc_gyr, src/fp_shared_core.c:993-1030 */
static double or_tacc_for_cap(const OrCtx *ctx, int model, double L, double dv, double cs,
                              double beta, double t_acc_direct)
{
    double mach;
    if (!(dv > 0.0) || !(L > 0.0) || !(cs > 0.0)) return 0.0;
    mach = dv / cs;
    if (mach < 0.0) mach = 0.0;
    if (ctx->par.mach_limit > 0.0 && mach > ctx->par.mach_limit) mach = ctx->par.mach_limit;
    if (mach <= 0.0) return 0.0;
    if (model == OR_DPP_ASA) {
        if (!(beta > 0.0)) return 0.0;
        return or_tacc_asa(ctx, L * K_MPC, cs, mach, beta);
    }
    if (model == OR_DPP_TTD) return or_tacc_ttd(ctx, L * K_MPC, cs, mach, dv);
    if (model == OR_DPP_DIRECT) return (t_acc_direct > 0.0 && isfinite(t_acc_direct)) ? t_acc_direct : 0.0;
    return 0.0;
}

/* fp_cr_energy_erg_cell, src/fp_shared_core.c:970-991 */
static double or_cr_energy(const OrCtx *ctx, const double *crp, const double *cre)
{
    const int n = ctx->nb;
    double e = 0.0;
    int j;
    if (crp != 0 && n > 4)
        for (j = 2; j < n - 2; j++) {
            const double ek = ctx->crp.E[j] - K_MP;
            if (ek > 0.0 && isfinite(crp[j])) e += ek * K_GEV * crp[j] * ctx->crp.dp[j];
        }
    if (cre != 0 && n > 4)
        for (j = 2; j < n - 2; j++) {
            const double ek = ctx->cre.E[j] - K_ME;
            if (ek > 0.0 && isfinite(cre[j])) e += ek * K_GEV * cre[j] * ctx->cre.dp[j];
        }
    return e;
}

/* fp_apply_eta_dpp_cap_cell, src/fp_shared_core.c:1032-1081 */
static void or_eta_cap(const OrCtx *ctx, int model, double L, double dv, double cs, double beta,
                       double mass, double t_acc_direct, const double *crp, const double *cre,
                       OrDpp *d)
{
    double tacc, ecr, qturb, eta, scale;
    int j;
    if (!(ctx->par.eta_dpp_cap > 0.0) || !isfinite(ctx->par.eta_dpp_cap)) return;
    if (!(mass > 0.0) || !(L > 0.0) || !(dv > 0.0)) return;
    if (crp == 0 && cre == 0) return;
    tacc = or_tacc_for_cap(ctx, model, L, dv, cs, beta, t_acc_direct);
    if (!(tacc > 0.0) || !isfinite(tacc)) return;
    ecr = or_cr_energy(ctx, crp, cre);
    qturb = 0.5 * mass * K_MSUN * dv * dv * dv / (L * K_MPC);
    if (!(ecr > 0.0) || !(qturb > 0.0) || !isfinite(ecr) || !isfinite(qturb)) return;
    eta = ecr / (qturb * tacc * K_GYR);
    if (!(eta > ctx->par.eta_dpp_cap) || !isfinite(eta)) return;
    scale = ctx->par.eta_dpp_cap / eta;
    for (j = 0; j < ctx->nb; j++) d->dpp[j] *= scale;
    for (j = 0; j < ctx->nb; j++) d->dppe[j] *= scale;
    d->m1 *= scale; d->p1 *= scale; d->em1 *= scale; d->ep1 *= scale;
}

/* prepare_momentumdiff_cell_major for one cell, src/fp_shared_core.c:1241-1317
 * with the models of src/FP_Coef.c:756-806. */
static void or_dpp_cell(const OrCtx *ctx, int model, double L, double dv, double cs, double beta,
                        double mass, double t_acc_direct, const double *crp, const double *cre,
                        OrDpp *d)
{
    const double epmax = 1.0e7;   /* tracer_fp_coef.c:262 */
    if (!(dv > 0.0) || !isfinite(dv) || model == OR_DPP_OFF) {
        or_dpp_off(ctx, d);
    } else if (model == OR_DPP_ASA) {
        const double mach = or_effective_mach(ctx, dv, cs);
        if (mach <= 0.0 || beta <= 0.0) or_dpp_off(ctx, d);
        else {
            const double t_acc = or_tacc_asa(ctx, L * K_MPC, cs, mach, beta);
            or_dpp_fill(ctx, 1.0 / ((2.0 + 2.0) * t_acc), epmax, d);
        }
    } else if (model == OR_DPP_TTD) {
        const double mach = or_effective_mach(ctx, dv, cs);
        if (mach <= 0.0 || dv <= 0.0) or_dpp_off(ctx, d);
        else {
            const double t_acc = or_tacc_ttd(ctx, L * K_MPC, cs, mach, dv);
            or_dpp_fill(ctx, 1.0 / ((2.0 + 2.0) * t_acc), epmax, d);
        }
    } else if (model == OR_DPP_DIRECT) {
        if (!(t_acc_direct > 0.0) || !isfinite(t_acc_direct)) or_dpp_off(ctx, d);
        else or_dpp_fill(ctx, 1.0 / (4.0 * t_acc_direct), epmax, d);
    } else {
        or_dpp_off(ctx, d);
    }
    if (model != OR_DPP_OFF)
        or_eta_cap(ctx, model, L, dv, cs, beta, mass, t_acc_direct, crp, cre, d);
}

/* ------------------------------------------------------------------ */
/* Chang-Cooper rows: src/Chang_Cooper.c:22-184 assembled as in        */
/* fp_build_cc_coeffs_from_terms, src/fp_shared_core.c:660-704         */
/* ------------------------------------------------------------------ */
static void or_face_weights(double w, double *delta, double *wp, double *wm)  /* :22-40 */
{
    *delta = 1.0 / w - 1.0 / (exp(w) - 1.0);
    if (fabs(w) < 0.1) {
        double den = 1.0 + pow(w, 2.0) / 24.0 + pow(w, 4.0) / 1920.0;
        *wp = exp(0.5 * w) / den;
        *wm = exp(-0.5 * w) / den;
    } else {
        double aw = fabs(w);
        double den = 1.0 - exp(-aw);
        *wp = aw * exp(-0.5 * aw + 0.5 * w) / den;
        *wm = aw * exp(-0.5 * aw - 0.5 * w) / den;
    }
}

static void or_face(double bl, double br, double cl, double cr, double xl, double xr,
                    double *delta, double *wp, double *wm, double *wout)      /* :42-64 */
{
    double w;
    *delta = 0.0; *wp = 0.0; *wm = 0.0;
    if (wout) *wout = 0.0;
    if (fabs(cl) <= 1.0e-200) return;
    w = 0.5 * (bl + br) / (0.5 * (cl + cr)) * (xr - xl);
    or_face_weights(w, delta, wp, wm);
    if (wout) *wout = w;
}

/* Builds a, b, c (positive coupling magnitudes) for one species:
 * rows b_i x_i - a_i x_{i-1} - c_i x_{i+1} = rhs_i.  Returns -1 on the NaN
 * conditions at which the reference exits (Chang_Cooper.c:166-183). */
static int or_build_cc(int n, double dt, const double *x, const double *dx,
                       const double *B, const double *C, const double *T,
                       double xm1, double xp1, double bm1, double bp1, double cm1, double cp1,
                       double *a, double *b, double *c, double *scratch)
{
    const int nm = n - 1;
    double *delta = scratch, *Wp = scratch + n, *Wm = scratch + 2 * n, *w = scratch + 3 * n;
    double Wpm1 = 0.0, Wmm1 = 0.0;
    int m;

    for (m = 0; m < nm; m++)
        or_face(B[m], B[m + 1], C[m], C[m + 1], x[m], x[m + 1], &delta[m], &Wp[m], &Wm[m], &w[m]);
    if (fabs(C[0]) > 1.0e-200)
        or_face(bm1, B[0], cm1, C[0], xm1, x[0], &delta[0], &Wpm1, &Wmm1, 0);
    or_face(B[nm], bp1, C[nm], cp1, x[nm], xp1, &delta[nm], &Wp[nm], &Wm[nm], &w[nm]);

    for (m = 1; m < nm; m++) {
        const double k = dt / (1.0 * dx[m]);
        if (fabs(C[m]) <= 1.0e-200) delta[m - 1] = 0.0;
        if (fabs(C[m]) > 1.0e-200) {             /* cc_build_interior_coeffs :66-104 */
            const double dxm_12 = x[m] - x[m - 1];
            const double dxm12 = x[m + 1] - x[m];
            const double cm_12 = 0.5 * (C[m] + C[m - 1]);
            const double cm12 = 0.5 * (C[m] + C[m + 1]);
            a[m] = k * cm_12 / dxm_12 * Wm[m - 1];
            b[m] = 1.0 + k * (cm_12 / dxm_12 * Wp[m - 1] + cm12 / dxm12 * Wm[m]) + dt / T[m];
            c[m] = k * cm12 / dxm12 * Wp[m];
        } else {
            const double d_12 = delta[m - 1], d12 = delta[m];
            const double bm_12 = 0.5 * (B[m] + B[m - 1]);
            const double bm12 = 0.5 * (B[m] + B[m + 1]);
            a[m] = -d_12 * bm_12 * dt / (1.0 * dx[m]);
            b[m] = 1.0 + k * ((1.0 - d_12) * bm_12 - d12 * bm12) + dt / T[m];
            c[m] = k * (1.0 - delta[m]) * bm12;
        }
    }
    {                                             /* cc_build_left_boundary :106-140 */
        const double k = dt / (1.0 * dx[0]);
        if (fabs(C[0]) > 1.0e-200) {
            const double c_12 = 0.0;
            a[0] = k * c_12 / (x[0] - xm1) * Wmm1;
            b[0] = 1.0 + k * (c_12 / (x[0] - xm1) * Wpm1 + 0.5 * (C[0] + C[1]) / (x[1] - x[0]) * Wm[0]) +
                   dt / T[0];
            c[0] = k * 0.5 * (C[0] + C[1]) / (x[1] - x[0]) * Wp[0];
        } else {
            const double b_12 = 0.0;
            a[0] = -delta[0] * b_12 * dt / (1.0 * dx[0]);
            b[0] = 1.0 + k * b_12 + dt / T[0];
            c[0] = k * (1.0 - delta[0]) * 0.5 * (B[0] + B[1]);
        }
    }
    {                                             /* cc_build_right_boundary :142-184 */
        const double k = dt / (1.0 * dx[nm]);
        if (fabs(C[nm]) > 1.0e-200) {
            a[nm] = k * (0.5 * (C[nm] + C[nm - 1])) / (x[nm] - x[nm - 1]) * Wm[nm - 1];
            b[nm] = 1.0 + k * ((0.5 * (C[nm] + C[nm - 1])) / (x[nm] - x[nm - 1]) * Wp[nm - 1]) + dt / T[nm];
            if (isnan(a[nm])) return -1;
            c[nm] = 0.0;
        } else {
            a[nm] = -delta[nm - 1] * 0.5 * (B[nm] + B[nm - 1]) * dt / (1.0 * dx[nm]);
            b[nm] = 1.0 + k * (0.5 * (B[nm - 1] + B[nm])) + dt / T[nm];
            c[nm] = 0.0;
        }
        if (isnan(c[nm])) return -1;
    }
    (void)w;
    return 0;
}

/* Coefficient terms of one species feeding the CC build:
 * prepare_cc_coeff_cell_major, src/fp_shared_core.c:2385-2427. */
static int or_cc_species(const OrGrid *g, int n, double dt, const double *radp,
                         const double *tloss, const double *dpp, double radpm1, double radpp1,
                         double dppm1, double dppp1, double *abc, double *scratch)
{
    double *B = scratch, *C = scratch + n;
    int j;
    for (j = 0; j < n; j++) {
        B[j] = radp[j] - 2.0 / g->p[j] * dpp[j];
        C[j] = dpp[j];
    }
    return or_build_cc(n, dt, g->p, g->dp, B, C, tloss, g->pm1, g->pp1,
                       radpm1 - 2.0 / g->pm1 * dppm1, radpp1 - 2.0 / g->pp1 * dppp1,
                       dppm1, dppp1, abc, abc + n, abc + 2 * n, scratch + 2 * n);
}

/* fp_thomas_solve_ws, src/fp_shared_core.c:226-257 */
static int or_thomas(int n, const double *a, const double *b, const double *c,
                     double *x, double *cp)
{
    int i;
    if (fabs(b[0]) <= 1.0e-300) return -2;
    cp[0] = -c[0] / b[0];
    x[0] /= b[0];
    for (i = 1; i < n; i++) {
        double den = b[i] + a[i] * cp[i - 1];
        if (fabs(den) <= 1.0e-300) return -2;
        cp[i] = (i == n - 1) ? 0.0 : -c[i] / den;
        x[i] = (x[i] + a[i] * x[i - 1]) / den;
    }
    for (i = n - 2; i >= 0; i--) x[i] -= cp[i] * x[i + 1];
    return 0;
}

/* ------------------------------------------------------------------ */
/* One cell, one segment: tracer_fp_cpu_evolve, src/tracer_fp_cpu.c:88-196 */
/* ------------------------------------------------------------------ */
typedef struct {
    double n_gas, kbt, b_field, divv, lturb, dv, cs, beta;
} OrBg;

typedef struct {
    double *ccp_on, *cce_on, *ccp_off, *cce_off;   /* [3][nb] each */
    double *radp_p, *tloss_p, *radp_e, *tloss_e;
    double *dpp_on, *dppe_on, *dpp_off, *dppe_off;
    double *inje, *cprime, *scratch;
} OrWs;

static OrWs or_ws_alloc(int n)
{
    OrWs w;
    double *blk = (double *)calloc((size_t)n * 36, sizeof(double));
    w.ccp_on = blk;            w.cce_on = blk + 3 * n;
    w.ccp_off = blk + 6 * n;   w.cce_off = blk + 9 * n;
    w.radp_p = blk + 12 * n;   w.tloss_p = blk + 13 * n;
    w.radp_e = blk + 14 * n;   w.tloss_e = blk + 15 * n;
    w.dpp_on = blk + 16 * n;   w.dppe_on = blk + 17 * n;
    w.dpp_off = blk + 18 * n;  w.dppe_off = blk + 19 * n;
    w.inje = blk + 20 * n;     w.cprime = blk + 21 * n;
    w.scratch = blk + 22 * n;  /* 14 n */
    return w;
}

static int or_cell_coeffs(const OrCtx *ctx, double dt, const OrBg *bg, const double *rad_ic,
                          double rad_ic_m1, double rad_ic_p1, double mass, int dis_adiab,
                          double t_acc_direct, const double *crp, const double *cre, OrWs *w)
{
    const int n = ctx->nb;
    const double divv_loss = dis_adiab ? 0.0 : bg->divv;
    double rpm1, rpp1, rem1, rep1;
    OrDpp on, off;
    int err = 0;

    or_crp_losses(ctx, bg->n_gas, bg->kbt, divv_loss, w->radp_p, w->tloss_p, &rpm1, &rpp1);
    or_cre_losses(ctx, bg->n_gas, bg->b_field, divv_loss, rad_ic, rad_ic_m1, rad_ic_p1,
                  w->radp_e, w->tloss_e, &rem1, &rep1);
    on.dpp = w->dpp_on; on.dppe = w->dppe_on;
    off.dpp = w->dpp_off; off.dppe = w->dppe_off;
    or_dpp_cell(ctx, ctx->par.dpp_model, bg->lturb, bg->dv, bg->cs, bg->beta, mass,
                t_acc_direct, crp, cre, &on);
    or_dpp_cell(ctx, OR_DPP_OFF, bg->lturb, bg->dv, bg->cs, bg->beta, mass,
                t_acc_direct, crp, cre, &off);
    err |= or_cc_species(&ctx->crp, n, dt, w->radp_p, w->tloss_p, on.dpp, rpm1, rpp1,
                         on.m1, on.p1, w->ccp_on, w->scratch);
    err |= or_cc_species(&ctx->cre, n, dt, w->radp_e, w->tloss_e, on.dppe, rem1, rep1,
                         on.em1, on.ep1, w->cce_on, w->scratch);
    err |= or_cc_species(&ctx->crp, n, dt, w->radp_p, w->tloss_p, off.dpp, rpm1, rpp1,
                         off.m1, off.p1, w->ccp_off, w->scratch);
    err |= or_cc_species(&ctx->cre, n, dt, w->radp_e, w->tloss_e, off.dppe, rem1, rep1,
                         off.em1, off.ep1, w->cce_off, w->scratch);
    return err ? -1 : 0;
}

/* prepare_secondary_sources_cell_major (transposed layout),
 * src/fp_shared_core.c:1591-1672 */
static void or_secondary(const OrCtx *ctx, double n_gas, const double *crp, const double *qepri,
                         double *inje)
{
    const int n = ctx->nb;
    int je, jp;
    for (je = 0; je < n; je++) inje[je] = 0.0;
    for (jp = ctx->fqe_jp0; jp < n; jp++) {
        const double nn = crp[jp];
        const double *wrow = ctx->fqe + (size_t)jp * n;
        for (je = 0; je < n; je++) inje[je] += nn * wrow[je];
    }
    for (je = 0; je < n; je++) {
        const double q = qepri ? qepri[je] : 0.0;
        inje[je] = inje[je] * K_GYR * n_gas + q;
    }
}

static int or_cell_segment(const OrCtx *ctx, int nstep, double dt, int windowed, int on_start,
                           int on_end, const OrBg *bg, const double *rad_ic, double rad_ic_m1,
                           double rad_ic_p1, const double *qpi, const double *qepri, double mass,
                           int dis_adiab, double t_acc_direct, double *crp, double *cre, OrWs *w)
{
    const int n = ctx->nb;
    int istep, j;
    if (or_cell_coeffs(ctx, dt, bg, rad_ic, rad_ic_m1, rad_ic_p1, mass, dis_adiab, t_acc_direct,
                       crp, cre, w) != 0)
        return -1;
    or_secondary(ctx, bg->n_gas, crp, qepri, w->inje);
    for (istep = 0; istep < nstep; istep++) {
        const int use_on = !windowed || (istep >= on_start && istep < on_end);
        const double *cp = use_on ? w->ccp_on : w->ccp_off;
        const double *ce = use_on ? w->cce_on : w->cce_off;
        for (j = 0; j < n; j++) crp[j] = dt * qpi[j] + crp[j];
        if (or_thomas(n, cp, cp + n, cp + 2 * n, crp, w->cprime) != 0) return -2;
        for (j = 0; j < n; j++) cre[j] = dt * w->inje[j] + cre[j];
        if (or_thomas(n, ce, ce + n, ce + 2 * n, cre, w->cprime) != 0) return -2;
    }
    return 0;
}

static OrBg or_bg_at(const double *bg, int ncell, int i)
{
    OrBg b;
    b.n_gas = bg[(size_t)OR_BG_NGAS * ncell + i];
    b.kbt = bg[(size_t)OR_BG_KBT * ncell + i];
    b.b_field = bg[(size_t)OR_BG_BFIELD * ncell + i];
    b.divv = bg[(size_t)OR_BG_DIVV * ncell + i];
    b.lturb = bg[(size_t)OR_BG_LTURB * ncell + i];
    b.dv = bg[(size_t)OR_BG_DV * ncell + i];
    b.cs = bg[(size_t)OR_BG_CS * ncell + i];
    b.beta = bg[(size_t)OR_BG_BETA * ncell + i];
    return b;
}

int or_cc_coeffs(const OrCtx *ctx, int ncell, double dt, const double *bg, const double *rad_ic,
                 const double *rad_ic_m1, const double *rad_ic_p1, const double *mass,
                 const unsigned char *dis, const double *crp_state, const double *cre_state,
                 double *ccp_on, double *cce_on, double *ccp_off, double *cce_off)
{
    const int n = ctx->nb;
    int err = 0, i;
    if (ctx == 0 || ncell <= 0) return -1;
    #pragma omp parallel for schedule(dynamic, 16) reduction(|:err)
    for (i = 0; i < ncell; i++) {
        OrWs w = or_ws_alloc(n);
        double *ric = w.scratch + 12 * n;   /* free tail of the scratch block */
        const OrBg b = or_bg_at(bg, ncell, i);
        size_t pn = (size_t)ncell * n;
        int j, k;
        for (j = 0; j < n; j++) ric[j] = rad_ic[(size_t)j * ncell + i];
        err |= or_cell_coeffs(ctx, dt, &b, ric, rad_ic_m1[i], rad_ic_p1[i], mass ? mass[i] : 0.0,
                              dis ? dis[i] : 0, ctx->par.t_acc_direct_gyr,
                              crp_state ? crp_state + (size_t)i * n : 0,
                              cre_state ? cre_state + (size_t)i * n : 0, &w);
        for (k = 0; k < 3; k++)
            for (j = 0; j < n; j++) {
                ccp_on[k * pn + (size_t)i * n + j] = w.ccp_on[k * n + j];
                cce_on[k * pn + (size_t)i * n + j] = w.cce_on[k * n + j];
                ccp_off[k * pn + (size_t)i * n + j] = w.ccp_off[k * n + j];
                cce_off[k * pn + (size_t)i * n + j] = w.cce_off[k * n + j];
            }
        free(w.ccp_on);
    }
    return err ? -1 : 0;
}

int or_evolve_segment(const OrCtx *ctx, int ncell, int nstep, double dt, int windowed,
                      int on_start, int on_end, const double *bg, const double *rad_ic,
                      const double *rad_ic_m1, const double *rad_ic_p1, const double *qpi,
                      const double *qepri, const double *mass, const unsigned char *dis,
                      double *crp_state, double *cre_state)
{
    const int n = ctx->nb;
    int err = 0, i;
    if (ctx == 0 || ncell <= 0) return -1;
    #pragma omp parallel for schedule(dynamic, 16) reduction(|:err)
    for (i = 0; i < ncell; i++) {
        OrWs w = or_ws_alloc(n);
        double *ric = (double *)malloc((size_t)n * sizeof(double));
        const OrBg b = or_bg_at(bg, ncell, i);
        int j;
        for (j = 0; j < n; j++) ric[j] = rad_ic[(size_t)j * ncell + i];
        if (or_cell_segment(ctx, nstep, dt, windowed, on_start, on_end, &b, ric, rad_ic_m1[i],
                            rad_ic_p1[i], qpi + (size_t)i * n, qepri + (size_t)i * n,
                            mass ? mass[i] : 0.0, dis ? dis[i] : 0, ctx->par.t_acc_direct_gyr,
                            crp_state + (size_t)i * n, cre_state + (size_t)i * n, &w) != 0)
            err = 1;
        free(ric);
        free(w.ccp_on);
    }
    return err ? -1 : 0;
}

/* ------------------------------------------------------------------ */
/* Sub-step estimator: src/tracer_fp_nsub.c:37-187, 242-282             */
/* ------------------------------------------------------------------ */
static double or_quantize_dt_sub(double t)         /* quantize_dt_sub :37-63 */
{
    static const double ladder[] = {1.0, 1.25, 1.6, 2.0, 2.5, 3.2, 4.0, 5.0, 6.4, 8.0};
    double e10, scale, norm, chosen = ladder[0];
    int i;
    if (!(t > 0.0) || !isfinite(t)) return t;
    e10 = floor(log10(t));
    scale = pow(10.0, e10);
    norm = t / scale;
    for (i = 0; i < 10; i++) {
        if (ladder[i] <= norm) chosen = ladder[i];
        else break;
    }
    return chosen * scale;
}

static double or_quantize_on_fraction(double f)    /* quantize_on_fraction :65-92 */
{
    static const double bins[] = {1.0 / 8.0, 1.0 / 4.0, 1.0 / 3.0, 1.0 / 2.0, 1.0};
    double chosen, best;
    int i;
    if (!(f > 0.0) || !isfinite(f)) return 1.0;
    if (f >= 1.0) return 1.0;
    chosen = bins[0];
    best = fabs(f - chosen);
    for (i = 1; i < 5; i++) {
        const double d = fabs(f - bins[i]);
        if (d < best) { chosen = bins[i]; best = d; }
    }
    return chosen;
}

int or_nsub(const OrCtx *ctx, int ntracer, double dt_snap, const double *bg,
            const double *rad_ic_row, int *nsub_out, int *target_out, int *non_out,
            unsigned char *capped)
{
    const int n = ctx->nb;
    int itr;
    if (ctx == 0 || ntracer <= 0 || dt_snap <= 0.0) return -1;
    for (itr = 0; itr < ntracer; itr++) {
        const double ng = bg[(size_t)OR_BG_NGAS * ntracer + itr];
        const double kbt = bg[(size_t)OR_BG_KBT * ntracer + itr];
        const double bf = bg[(size_t)OR_BG_BFIELD * ntracer + itr];
        const double dvv = bg[(size_t)OR_BG_DIVV * ntracer + itr];
        const double lt = bg[(size_t)OR_BG_LTURB * ntracer + itr];
        const double dv = bg[(size_t)OR_BG_DV * ntracer + itr];
        /* endpoint loss prepass :242-282 */
        const double p_lo = or_b_coulomb_p(ng, ctx->crp.p[0], kbt) + 1.0 / 3.0 * dvv * ctx->crp.p[0];
        const double p_hi = or_b_coulomb_p(ng, ctx->crp.p[n - 1], kbt) + 1.0 / 3.0 * dvv * ctx->crp.p[n - 1];
        const double e_lo = or_b_synch(ctx->cre.p[0], bf) + rad_ic_row[0] +
                            or_b_coulomb_e(ng, ctx->cre.p[0]) + 1.0 / 3.0 * dvv * ctx->cre.p[0];
        const double e_hi = or_b_synch(ctx->cre.p[n - 1], bf) + rad_ic_row[n - 1] +
                            or_b_coulomb_e(ng, ctx->cre.p[n - 1]) + 1.0 / 3.0 * dvv * ctx->cre.p[n - 1];
        /* compute_nsubsteps_core :94-187 */
        const double te0 = ctx->cre.p[0] / e_lo;
        const double tp0 = ctx->crp.p[0] / p_lo;
        const double teN = ctx->cre.p[n - 1] / e_hi;
        const double tpN = ctx->crp.p[n - 1] / p_hi;
        const double tmin = fmin(fabs(tp0), fmin(fabs(teN), fmin(fabs(te0), fabs(tpN))));
        double target = dt_snap / 10.0, used, tn, raw, onf = 1.0;
        int nsub, non;
        if (isfinite(tmin) && tmin > 0.0) {
            const double stab = ctx->par.nsub_safety * tmin;
            if (stab < target) target = stab;
        }
        if (target <= 0.0 || !isfinite(target)) target = dt_snap / 10.0;
        tn = ceil(dt_snap / target);
        if (!isfinite(tn) || tn > 1000000.0) tn = 1000000.0;
        if (tn < 10.0) tn = 10.0;
        used = or_quantize_dt_sub(target);
        if (!(used > 0.0) || !isfinite(used) || used > target) used = target;
        raw = ceil(dt_snap / used);
        if (!isfinite(raw) || raw > 1000000.0) raw = 1000000.0;
        if (raw < 10.0) raw = 10.0;
        nsub = (int)raw;
        if (capped) capped[itr] = 0;
        if (ctx->par.nsub_max > 0 && nsub > ctx->par.nsub_max) {
            nsub = ctx->par.nsub_max;
            if (capped) capped[itr] = 1;
        }
        if (ctx->par.reacc_window_mode == 1 && ctx->par.f_eddy > 0.0 && dv > 0.0) {
            const double t_eddy = lt * 3.0857e24 / dv / 3.1536e16;
            if (ctx->par.f_eddy * t_eddy < dt_snap)
                onf = or_quantize_on_fraction(ctx->par.f_eddy * t_eddy / dt_snap);
        }
        non = (int)floor((double)nsub * onf + 0.5);
        if (non < 1) non = 1;
        if (non > nsub) non = nsub;
        nsub_out[itr] = nsub;
        if (target_out) target_out[itr] = (int)tn;
        non_out[itr] = non;
    }
    return 0;
}

/* tracer_bucket_build_snapshot, src/tracer_fp_bucket.c:208-262 */
int or_buckets(int ntracer, const int *nsub, const int *non, int *bucket_ids, int *indices,
               int *steps, int *onsteps, int *offsets, int *counts, int *nbuckets_out)
{
    int itr, ib, nb = 0, off = 0;
    int *wr = (int *)calloc((size_t)ntracer, sizeof(int));
    for (itr = 0; itr < ntracer; itr++) counts[itr] = 0;
    for (itr = 0; itr < ntracer; itr++) {
        int id = -1;
        for (ib = 0; ib < nb; ib++)
            if (steps[ib] == nsub[itr] && onsteps[ib] == non[itr]) { id = ib; break; }
        if (id < 0) { id = nb; steps[id] = nsub[itr]; onsteps[id] = non[itr]; nb++; }
        bucket_ids[itr] = id;
        counts[id]++;
    }
    for (ib = 0; ib < nb; ib++) { offsets[ib] = off; wr[ib] = off; off += counts[ib]; }
    for (itr = 0; itr < ntracer; itr++) indices[wr[bucket_ids[itr]]++] = itr;
    *nbuckets_out = nb;
    free(wr);
    return 0;
}

/* tracer_fp_choose_coeff_interp_segments, src/tracer_fp_setup.c:73-95 */
int or_coeff_segments(const OrCtx *ctx, int nsub, int allow_interp)
{
    int seg = 1, max_allowed, max_seg = ctx->par.coeff_interp_max_segments;
    if (!allow_interp || nsub <= 1) return 1;
    if (ctx->par.coeff_interp_min_steps <= 0) return 1;
    if (max_seg < 1) max_seg = 1;
    max_allowed = nsub / ctx->par.coeff_interp_min_steps;
    if (max_allowed < 1) return 1;
    while (seg <= 1073741823 && seg * 2 <= max_seg && seg * 2 <= max_allowed) seg *= 2;
    if (seg > nsub) seg = nsub;
    if (seg < 1) seg = 1;
    return seg;
}

/* interp_array element, src/tracer_fp_batch.c:89-111 */
static double or_lerp(double cur, double nxt, double alpha)
{
    if (alpha <= 0.0) return cur;
    if (alpha >= 1.0) return nxt;
    return cur + alpha * (nxt - cur);
}

/*
 * One tracer through one snapshot, as tracer_fp_batch_execute_bucket
 * (src/tracer_fp_batch.c:651-827) runs a bucket of one: segments with
 * interpolated backgrounds, the centred reacceleration window, and the
 * direct-t_acc schedule (cpu_direct_tacc_value, :44-62).
 */
static int or_tracer_snapshot(const OrCtx *ctx, int nsub, int non, int allow_interp,
                              double dt_snap, double elapsed, const OrBg *cur, const OrBg *nxt,
                              const double *ic_cur, const double *ic_nxt, const double *qpi,
                              const double *qepri, double mass, int dis, double *crp, double *cre,
                              OrWs *w, double *ric)
{
    const int n = ctx->nb;
    const int nseg = or_coeff_segments(ctx, nsub, allow_interp);
    const int on_start = (nsub - non) / 2, on_end = on_start + non;
    const double base_dt = dt_snap / (double)nsub;
    int iseg, j;

    for (iseg = 0; iseg < nseg; iseg++) {
        const double alpha = (nseg > 1) ? ((double)iseg + 0.5) / (double)nseg : 0.0;
        const int b = (int)(((long long)iseg * nsub) / nseg);
        const int e = (int)(((long long)(iseg + 1) * nsub) / nseg);
        const int steps = e - b;
        OrBg bg = *cur;
        double m1 = ic_cur[n], p1 = ic_cur[n + 1], tacc;
        int sob, soe, windowed, sl, el;
        if (steps <= 0) continue;
        for (j = 0; j < n; j++) ric[j] = ic_cur[j];
        if (nseg > 1) {
            bg.n_gas = or_lerp(cur->n_gas, nxt->n_gas, alpha);
            bg.kbt = or_lerp(cur->kbt, nxt->kbt, alpha);
            bg.b_field = or_lerp(cur->b_field, nxt->b_field, alpha);
            bg.divv = or_lerp(cur->divv, nxt->divv, alpha);
            bg.lturb = or_lerp(cur->lturb, nxt->lturb, alpha);
            bg.dv = or_lerp(cur->dv, nxt->dv, alpha);
            bg.cs = or_lerp(cur->cs, nxt->cs, alpha);
            bg.beta = or_lerp(cur->beta, nxt->beta, alpha);
            for (j = 0; j < n; j++) ric[j] = or_lerp(ic_cur[j], ic_nxt[j], alpha);
            m1 = or_lerp(ic_cur[n], ic_nxt[n], alpha);
            p1 = or_lerp(ic_cur[n + 1], ic_nxt[n + 1], alpha);
        }
        sob = (on_start > b) ? on_start : b;
        soe = (on_end < e) ? on_end : e;
        if (soe < sob) soe = sob;
        windowed = ((soe - sob) < steps) ? 1 : 0;
        sl = sob - b;
        el = sl + (soe - sob);
        tacc = ctx->par.t_acc_direct_gyr;
        if (ctx->par.dpp_model == OR_DPP_DIRECT && isfinite(tacc) && tacc > 0.0 &&
            isfinite(ctx->par.t_off_gyr) && ctx->par.t_off_gyr > 0.0 &&
            isfinite(ctx->par.t_acc_off_gyr) && ctx->par.t_acc_off_gyr > 0.0) {
            const double tmid = elapsed + ((double)b + 0.5 * (double)steps) * base_dt;
            if (tmid < ctx->par.t_off_gyr) tacc = ctx->par.t_acc_off_gyr;
        }
        if (or_cell_segment(ctx, steps, dt_snap / (double)nsub, windowed, sl, el, &bg, ric, m1, p1,
                            qpi, qepri, mass, dis, tacc, crp, cre, w) != 0)
            return -1;
    }
    return 0;
}

int or_snapshot_with_ic(const OrCtx *ctx, int ntracer, const double *bg_curr, const double *bg_next,
                        const double *ic_curr, const double *ic_next, int allow_interp,
                        double dt_snap, double elapsed, const double *qpi, const double *qepri,
                        const double *mass, const unsigned char *dis, double *crp_state,
                        double *cre_state, int *nsub_out, int *non_out, int *bucket_ids_out,
                        int *nbuckets_out)
{
    const int n = ctx->nb;
    const double *bn = allow_interp ? bg_next : bg_curr;
    const double *icn = allow_interp ? ic_next : ic_curr;
    int *nsub = (int *)calloc((size_t)ntracer * 8, sizeof(int));
    int *non = nsub + ntracer, *bid = nsub + 2 * (size_t)ntracer, *idx = nsub + 3 * (size_t)ntracer;
    int *steps = nsub + 4 * (size_t)ntracer, *ons = nsub + 5 * (size_t)ntracer;
    int *offs = nsub + 6 * (size_t)ntracer, *cnts = nsub + 7 * (size_t)ntracer;
    int nb = 0, err = 0, i;

    if (nsub == 0) return -3;
    if (or_nsub(ctx, ntracer, dt_snap, bg_curr, ic_curr, nsub, 0, non, 0) != 0) { free(nsub); return -1; }
    or_buckets(ntracer, nsub, non, bid, idx, steps, ons, offs, cnts, &nb);

    #pragma omp parallel for schedule(dynamic, 8) reduction(|:err)
    for (i = 0; i < ntracer; i++) {
        OrWs w = or_ws_alloc(n);
        double *ric = (double *)malloc((size_t)n * sizeof(double));
        const OrBg cur = or_bg_at(bg_curr, ntracer, i);
        const OrBg nxt = or_bg_at(bn, ntracer, i);
        if (or_tracer_snapshot(ctx, nsub[i], non[i], allow_interp, dt_snap, elapsed, &cur, &nxt,
                               ic_curr, icn, qpi + (size_t)i * n, qepri + (size_t)i * n,
                               mass ? mass[i] : 0.0, dis ? dis[i] : 0,
                               crp_state + (size_t)i * n, cre_state + (size_t)i * n, &w, ric) != 0)
            err = 1;
        free(ric);
        free(w.ccp_on);
    }
    if (nsub_out) memcpy(nsub_out, nsub, (size_t)ntracer * sizeof(int));
    if (non_out) memcpy(non_out, non, (size_t)ntracer * sizeof(int));
    if (bucket_ids_out) memcpy(bucket_ids_out, bid, (size_t)ntracer * sizeof(int));
    if (nbuckets_out) *nbuckets_out = nb;
    free(nsub);
    return err ? -1 : 0;
}

int or_snapshot(const OrCtx *ctx, int ntracer, const double *bg_curr, const double *bg_next,
                double z_curr, double z_next, int allow_interp, double dt_snap, double elapsed,
                const double *qpi, const double *qepri, const double *mass,
                const unsigned char *dis, double *crp_state, double *cre_state, int *nsub_out,
                int *non_out, int *bucket_ids_out, int *nbuckets_out)
{
    const int n = ctx->nb;
    double *ic = (double *)malloc((size_t)(n + 2) * 2 * sizeof(double));
    int err;
    if (ic == 0) return -3;
    or_ic_row(ctx, z_curr, ic, ic + n, ic + n + 1);
    if (allow_interp) or_ic_row(ctx, z_next, ic + n + 2, ic + 2 * n + 2, ic + 2 * n + 3);
    else memcpy(ic + n + 2, ic, (size_t)(n + 2) * sizeof(double));
    err = or_snapshot_with_ic(ctx, ntracer, bg_curr, bg_next, ic, ic + n + 2, allow_interp, dt_snap,
                              elapsed, qpi, qepri, mass, dis, crp_state, cre_state, nsub_out, non_out,
                              bucket_ids_out, nbuckets_out);
    free(ic);
    return err;
}

/* ------------------------------------------------------------------ */
/* Context                                                             */
/* ------------------------------------------------------------------ */
OrCtx *or_create(const OrParams *par)
{
    OrCtx *ctx;
    int n;
    double *blk;
    if (par == 0 || par->nb < 8) return 0;
    n = par->nb;
    ctx = (OrCtx *)calloc(1, sizeof(OrCtx));
    if (ctx == 0) return 0;
    ctx->par = *par;
    ctx->nb = n;
    blk = (double *)calloc((size_t)n * 14 + (size_t)n * n, sizeof(double));
    ctx->crp.p = blk;          ctx->crp.dp = blk + n;      ctx->crp.E = blk + 2 * n;
    ctx->cre.p = blk + 3 * n;  ctx->cre.dp = blk + 4 * n;  ctx->cre.E = blk + 5 * n;
    ctx->beta_p = blk + 6 * n;
    ctx->crp_p2 = blk + 7 * n; ctx->crp_exp_cut = blk + 8 * n;
    ctx->crp_sigma_pp = blk + 9 * n; ctx->crp_sigmoid_pp = blk + 10 * n;
    ctx->cre_p2 = blk + 11 * n; ctx->cre_exp_cut = blk + 12 * n;
    ctx->fqe = blk + 14 * n;
    ctx->np_min_qe = (int *)calloc((size_t)n, sizeof(int));
    or_build_grid(ctx);
    or_build_grid_cache(ctx);
    or_build_secondary_kernel(ctx);
    return ctx;
}

void or_destroy(OrCtx *ctx)
{
    if (ctx == 0) return;
    free(ctx->crp.p);
    free(ctx->np_min_qe);
    free(ctx);
}

int or_get_grid(const OrCtx *ctx, int species, double *out)
{
    const OrGrid *g = (species == 0) ? &ctx->crp : &ctx->cre;
    const int n = ctx->nb;
    memcpy(out, g->p, (size_t)n * sizeof(double));
    memcpy(out + n, g->dp, (size_t)n * sizeof(double));
    memcpy(out + 2 * n, g->E, (size_t)n * sizeof(double));
    out[3 * n] = g->pm1;
    out[3 * n + 1] = g->pp1;
    return 0;
}

int or_get_beta_p(const OrCtx *ctx, double *out)
{
    memcpy(out, ctx->beta_p, (size_t)ctx->nb * sizeof(double));
    return 0;
}

int or_get_pp_cache(const OrCtx *ctx, double *sigma_pp, double *sigmoid_pp, int *j_pp)
{
    if (sigma_pp) memcpy(sigma_pp, ctx->crp_sigma_pp, (size_t)ctx->nb * sizeof(double));
    if (sigmoid_pp) memcpy(sigmoid_pp, ctx->crp_sigmoid_pp, (size_t)ctx->nb * sizeof(double));
    if (j_pp) *j_pp = ctx->crp_j_pp;
    return 0;
}

int or_get_secondary_kernel(const OrCtx *ctx, double *fqe_flat, int *np_min_qe)
{
    if (fqe_flat) memcpy(fqe_flat, ctx->fqe, (size_t)ctx->nb * ctx->nb * sizeof(double));
    if (np_min_qe) memcpy(np_min_qe, ctx->np_min_qe, (size_t)ctx->nb * sizeof(int));
    return 0;
}

void or_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
