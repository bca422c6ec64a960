/*
 * croma_oracle_dsa.c -- CPU restatement of the reference's per-snapshot DSA
 * (diffusive shock acceleration) injection into tracer spectra.
 *
 * Test infrastructure only (the checker): it is linked into
 * oracle/_build/liboracle.so and is never part of the product.  Each
 * function restates the reference routine named beside it
 * (kosukenishiwaki/croma-fp sources):
 *
 *   shock inputs          tracer_dsa_resolve_tracer_input   src/tracer_fp_dsa.c:26-108
 *   efficiency models     g_dsa_models / dsa_eta_model      src/DSA_MODELS.c:262-468
 *   compression, slope    dsa_compression_ratio / _slope    src/DSA_MODELS.c:524-561
 *   injection momenta     dsa_thermal_momentum_mc ...       src/DSA_MODELS.c:599-650
 *   proton normalisation  dsa_proton_edens_unit (Simpson)   src/DSA_MODELS.c:690-776
 *   electron normalisation dsa_electron_norm_from_kep_at_pinj_p src/DSA_MODELS.c:1022-1070
 *   DSA grid              dsa_init_grid / _fill_grid1d      src/DSA_MODELS.c:221-300, 1191-1261
 *   source on the grid    dsa_spectrum_f / _dp              src/DSA_MODELS.c:1396-1438
 *   reacceleration        tracer_fp_dsa_reacc.c:60-236
 *   per-tracer driver     tracer_fp_apply_dsa_tracer_injection_snapshot
 *                                                           src/tracer_fp_dsa.c:184-565
 *
 * State arrays are cell-major [ntracer][nb], as in the reference.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "croma_oracle.h"

#define DSA_MP_G 1.67262192369e-24
#define DSA_ME_G 9.1093837015e-28
#define DSA_KB_CGS 1.380649e-16
#define DSA_C_EXACT 2.99792458e10    /* speed of light of the DSA model code */
#define DSA_C_CROMA 2.999e10         /* CROMA's c (CONSTANTS.c), used by the tracer energies */
#define DSA_4PI 12.566370614359172
#define DSA_MSUN 1.99e33
#define DSA_PI 3.14159265358979323846

/* ---- acceleration efficiency models: a quartic in (M - 1) over M^4 with a
 * family-specific low-Mach branch and ceiling ---- */
typedef struct {
    int family;      /* 0 KR07, 1 KR13, 2 Ryu19 */
    int reacc;       /* 0 initial, 1 reacceleration */
    double xcr0;
    double b[5];
    double mach_crit;
    double scale;
} DsaModel;

static const DsaModel kModels[8] = {
    {0, 0, 0.0, {5.46, -9.78, 4.17, -0.33, 0.57}, 1.0, 1.0},            /* KR07 */
    {0, 1, 0.3, {0.24, -1.56, 2.8, 0.512, 0.557}, 1.0, 1.0},            /* KR07r */
    {1, 0, 0.0, {-2.87, 9.67, -8.88, 1.94, 0.18}, 2.0, 1.0},            /* KR13 */
    {1, 1, 0.05, {-0.72, 2.73, -3.29, 1.34, 0.19}, 2.0, 1.0},           /* KR13r */
    {1, 0, 0.0, {-2.87, 9.67, -8.88, 1.94, 0.18}, 2.0, 0.5},            /* CS14 */
    {1, 1, 0.05, {-0.72, 2.73, -3.29, 1.34, 0.19}, 2.0, 0.5},           /* CS14r */
    {2, 0, 0.0, {-1.5255, 2.4026, -1.2534, 0.2215, 0.0336}, 2.25, 1.0}, /* Ryu19 */
    {2, 1, 0.05, {0.3965, -0.21898, -0.2074, 0.1319, 0.0351}, 2.25, 1.0} /* Ryu19r */
};

static double quartic_over_m4(double m, const double b[5])
{
    if (m <= 0.0) return 0.0;
    const double x = m - 1.0;
    return (b[0] + b[1] * x + b[2] * x * x + b[3] * x * x * x + b[4] * x * x * x * x) / (m * m * m * m);
}

static double dsa_eta(double m, int id)
{
    if (id < 0 || id >= 8) return 0.0;
    const DsaModel *md = &kModels[id];
    if (m < md->mach_crit) return 0.0;
    const double poly = quartic_over_m4(m, md->b);
    double eta;
    if (md->family == 0 && !md->reacc) {
        eta = (m <= 2.0) ? 1.96e-3 * (m * m - 1.0) : poly;
    } else if (md->family == 0) {
        if (m <= 1.5) {
            const double g = 5.0 / 3.0, m2 = m * m;
            const double xs = (g + 1.0) / (g - 1.0 + 2.0 / m2);
            const double d0 = 2.0 * (((2.0 * g * m2 - g + 1.0) / (g + 1.0)) - pow(xs, g)) /
                              (g * (g - 1.0) * m2 * xs);
            eta = 1.025 * d0;
        } else {
            eta = poly;
        }
    } else if (md->family == 1 && !md->reacc) {
        if (m <= 5.0) eta = -0.0005950569221922047 + 1.880258286365841e-5 * pow(m, 5.334076006529829);
        else if (m <= 15.0) eta = poly;
        else eta = 0.21152;
    } else if (md->family == 1) {
        eta = (m <= 17.7) ? poly : 0.2055;
    } else {
        eta = (m <= 34.0) ? poly : 0.0348;
    }
    eta *= md->scale;
    return eta < 0.0 ? 0.0 : eta;
}

static double compression_ratio(double m, double g)
{
    if (m <= 1.0 || g <= 1.0) return 1.0;
    const double m2 = m * m;
    const double den = (g - 1.0) * m2 + 2.0;
    if (den <= 0.0) return 1.0;
    return (g + 1.0) * m2 / den;
}

static double slope_d3p(double m, double g)
{
    if (m <= 1.0) return 0.0;
    const double r = compression_ratio(m, g);
    if (r <= 1.0) return 0.0;
    return 3.0 * r / (r - 1.0);
}

static double injection_momentum(double temp, double chi, double mass_g)
{
    if (chi <= 0.0 || temp <= 0.0) return 0.0;
    const double th = 2.0 * DSA_KB_CGS * temp / (mass_g * DSA_C_EXACT * DSA_C_EXACT);
    if (th <= 0.0) return 0.0;
    return chi * sqrt(th);
}

/* (p / p_inj)^-q exp(-(p / p_max)^2) with the exponent clamped to +-700 */
static double spectrum_shape(double p, double pinj, double q, double pmax)
{
    if (p <= 0.0 || pinj <= 0.0 || pmax <= 0.0 || p < pinj) return 0.0;
    const double rm = p / pmax;
    double e = -rm * rm;
    if (e < -700.0) e = -700.0;
    if (e > 700.0) e = 700.0;
    return pow(p / pinj, -q) * exp(e);
}

/* 4 pi m_p c^2 int_{p_inj}^{p_max} (sqrt(1+p^2) - 1) p^2 shape dp, composite
 * Simpson with nstep intervals */
static double proton_edens_unit(double pinj, double q, double pmax, int nstep)
{
    if (pinj <= 0.0 || pmax <= 0.0 || pmax <= pinj) return 0.0;
    if (nstep < 2) nstep = 2000;
    if (nstep % 2) nstep++;
    const double h = (pmax - pinj) / (double)nstep;
#define INTEGRAND(pp) (((pp) <= 0.0 || (pp) < pinj) ? 0.0 : \
        (sqrt(1.0 + (pp) * (pp)) - 1.0) * (pp) * (pp) * spectrum_shape((pp), pinj, q, pmax))
    double s = INTEGRAND(pinj) + INTEGRAND(pmax);
    for (int i = 1; i < nstep; i++) {
        const double p = pinj + h * (double)i;
        s += ((i % 2) ? 4.0 : 2.0) * INTEGRAND(p);
    }
#undef INTEGRAND
    return DSA_4PI * DSA_MP_G * DSA_C_EXACT * DSA_C_EXACT * (s * h / 3.0);
}

/* DSA grid momenta at the FP bins: the DSA grid extends the FP grid's
 * log-spacing down to pmin_dsa and recomputes p = 10^(pmin + j dlogp). */
static void dsa_grid_p(const double *p_fp, int nb, double pmin_dsa_log10, double *out)
{
    const double dlogp = log10(p_fp[1]) - log10(p_fp[0]);
    const double pmin_fp = log10(p_fp[0]);
    int extra = 0;
    if (dlogp > 0.0 && pmin_dsa_log10 < pmin_fp) {
        extra = (int)ceil((pmin_fp - pmin_dsa_log10) / dlogp - 1.0e-12);
        if (extra < 0) extra = 0;
    }
    const double pmin_grid = pmin_fp - dlogp * (double)extra;
    for (int j = 0; j < nb; j++) out[j] = pow(10.0, pmin_grid + dlogp * (double)(j + extra));
}

/* 4 pi p^2 A (p/p_inj)^-q exp(-(p/p_max)^2) on [p_inj, p_max], else 0 */
static double source_dp(double A, double pinj, double q, double pmax, double p)
{
    if (p <= 0.0 || p < pinj || p > pmax) return 0.0;
    const double f = A * pow(p / pinj, -q) * exp(-(p / pmax) * (p / pmax));
    if (f <= 0.0) return 0.0;
    return DSA_4PI * p * p * f;
}

static double ekin_erg(double p, int electron)
{
    const double m = electron ? DSA_ME_G : DSA_MP_G;
    return m * DSA_C_CROMA * DSA_C_CROMA * (sqrt(1.0 + p * p) - 1.0);
}

static double edens_from_state(const double *p, const double *dp, const double *state, int nb,
                               double volume, double pmin, int electron)
{
    if (!(volume > 0.0)) return 0.0;
    double e = 0.0;
    for (int j = 0; j < nb; j++) {
        if (p[j] < pmin) continue;
        e += ekin_erg(p[j], electron) * state[j] * dp[j];
    }
    return e / volume;
}

/* ---- reacceleration deltas (tracer_fp_dsa_reacc.c) ---- */
static double reacc_positive(const double *p, const double *dp, const double *state, int nb,
                             double vdown, double q, double pmin, double *delta, int electron)
{
    double integral = 0.0, de = 0.0;
    for (int j = 0; j < nb; j++) delta[j] = 0.0;
    if (!(vdown > 0.0) || !(q > 0.0)) return 0.0;
    for (int j = (nb > 1 ? 1 : 0); j < nb; j++) {
        if (!(p[j] > 0.0) || p[j] < pmin) continue;
        const double cur = state[j] / vdown;
        const double fpre = cur / (4.0 * DSA_PI * p[j] * p[j]);
        integral += pow(p[j], q - 1.0) * fpre * dp[j];
        const double re = 4.0 * DSA_PI * p[j] * p[j] * q * pow(p[j], -q) * integral;
        if (re > cur) {
            delta[j] = re - cur;
            de += ekin_erg(p[j], electron) * delta[j] * dp[j];
        }
    }
    return de;
}

static double reacc_convolution(const double *p, const double *dp, const double *state, int nb,
                                double vup, double vdown, double q, double pmin, double *delta,
                                int electron)
{
    double integral = 0.0, de = 0.0;
    for (int j = 0; j < nb; j++) delta[j] = 0.0;
    if (!(vup > 0.0) || !(vdown > 0.0) || !(q > 0.0)) return 0.0;
    const double alpha = q - 2.0;
    for (int j = (nb > 1 ? 1 : 0); j < nb; j++) {
        if (!(p[j] > 0.0)) continue;
        const double seed = state[j] / vup, cur = state[j] / vdown;
        if (p[j] < pmin) continue;
        integral += pow(p[j], alpha - 1.0) * seed * dp[j];
        double d = (alpha + 2.0) * pow(p[j], -alpha) * integral - cur;
        if (!isfinite(d)) continue;
        if (d < -cur) d = -cur;
        delta[j] = d;
        de += ekin_erg(p[j], electron) * d * dp[j];
    }
    return de;
}

static double delta_edens(const double *p, const double *dp, const double *delta, int nb, double pmin,
                          int electron)
{
    if (nb <= 4) return 0.0;
    double e = 0.0;
    for (int j = 2; j <= nb - 3; j++) {
        if (!(p[j] > 0.0) || p[j] < pmin) continue;
        if (!isfinite(delta[j])) continue;
        e += ekin_erg(p[j], electron) * delta[j] * dp[j];
    }
    return e;
}

static double interp_lin(const double *p, const double *dens, int nb, double x)
{
    if (nb <= 2 || !(x > 0.0)) return 0.0;
    int lo = 1, hi = nb - 2;
    if (x < p[lo] || x > p[hi]) return 0.0;
    while (hi - lo > 1) {
        const int mid = lo + (hi - lo) / 2;
        if (p[mid] <= x) lo = mid;
        else hi = mid;
    }
    if (p[hi] <= p[lo]) return dens[lo];
    return dens[lo] + (dens[hi] - dens[lo]) * (x - p[lo]) / (p[hi] - p[lo]);
}

static double reacc_adiabatic(const double *p, const double *dp, const double *state, int nb,
                              double vup, double vdown, double ratio, double pmin, double *delta,
                              double *scratch, int electron)
{
    if (!(vup > 0.0) || !(vdown > 0.0) || !(ratio > 0.0) || !isfinite(ratio)) {
        for (int j = 0; j < nb; j++) delta[j] = 0.0;
        return 0.0;
    }
    const double shift = cbrt(ratio), norm = shift * shift;
    for (int j = 0; j < nb; j++) {
        scratch[j] = state[j] / vup;
        delta[j] = 0.0;
    }
    for (int j = 0; j < nb; j++) {
        if (!(p[j] > 0.0) || p[j] < pmin) continue;
        const double cur = state[j] / vdown;
        const double ad = norm * interp_lin(p, scratch, nb, p[j] / shift);
        if (!isfinite(cur) || !isfinite(ad)) continue;
        delta[j] = ad - cur;
    }
    return delta_edens(p, dp, delta, nb, pmin, electron);
}

/* tracer_dsa_resolve_tracer_input: the upstream state of one tracer */
static int resolve_input(const OrDsaParams *prm, const OrShockFields *sh, int t, double density_unit,
                         double *mach, double *temp, double *rho1, double *u1)
{
    if (sh->has_dsa) {
        if (!sh->dsa_trigger || !sh->dsa_mach || !sh->dsa_pre_density || !sh->dsa_flux_cgs) return 0;
        if (!(sh->dsa_trigger[t] > 0.5)) return 0;
        const double flux = sh->dsa_flux_cgs[t];
        const double m = sh->dsa_mach[t];
        const double r = sh->dsa_pre_density[t] * density_unit;
        if (!(m >= prm->min_mach) || !isfinite(m) || !(r > 0.0) || !isfinite(r)) return 0;
        if (!(flux > 0.0) || !isfinite(flux)) return 0;
        const double u = cbrt(2.0 * flux / r);
        if (!(u > 0.0) || !isfinite(u)) return 0;
        const double T = (prm->mu_mol * DSA_MP_G / (prm->gamma_gas * DSA_KB_CGS)) * (u * u) / (m * m);
        if (!(T > 0.0) || !isfinite(T)) return 0;
        *mach = m; *temp = T; *rho1 = r; *u1 = u;
        return 1;
    }
    if (!sh->mach || !sh->prestemp || !sh->presden) return 0;
    const double m = sh->mach[t], T = sh->prestemp[t];
    if (!(m >= prm->min_mach) || !(T > 0.0) || !isfinite(m) || !isfinite(T)) return 0;
    if (sh->shock_side_code) {
        const int side = (int)floor(sh->shock_side_code[t] + 0.5);
        if (side == -1 || side == 99) return 0;
    }
    const double r = (sh->pre_density_cgs && sh->pre_density_cgs[t] > 0.0)
                   ? sh->pre_density_cgs[t] : sh->presden[t] * density_unit;
    if (!(r > 0.0) || !isfinite(r)) return 0;
    const double u = (sh->upstream_speed_cgs && sh->upstream_speed_cgs[t] > 0.0)
                   ? sh->upstream_speed_cgs[t]
                   : m * sqrt(prm->gamma_gas * DSA_KB_CGS * T / (prm->mu_mol * DSA_MP_G));
    if (!(u > 0.0) || !isfinite(u)) return 0;
    *mach = m; *temp = T; *rho1 = r; *u1 = u;
    return 1;
}

int or_dsa_inject(const OrDsaParams *prm, int nb, const double *p_p, const double *dp_p,
                  const double *p_e, const double *dp_e, const OrShockFields *sh, int ntracer,
                  const double *mass_msun, double density_unit, double dt_gyr, int mode,
                  int reacc_mode, double *crp, double *cre, double *qpi, double *qepri,
                  unsigned char *dis, int *ninjected)
{
    if (ninjected) *ninjected = 0;
    if (!prm || !sh || ntracer <= 0 || !mass_msun || mode == OR_DSA_OFF) return 0;
    if ((mode == OR_DSA_STATE || mode == OR_DSA_SOURCE || reacc_mode != OR_REACC_OFF) && (!crp || !cre))
        return -1;
    if (mode == OR_DSA_SOURCE && (!qpi || !qepri || !(dt_gyr > 0.0) || !isfinite(dt_gyr))) return -1;
    if (mode != OR_DSA_STATE && mode != OR_DSA_SOURCE) return 0;

    const double chi_e = (prm->chi_e > 0.0) ? prm->chi_e : prm->chi_p;
    const int inj_p = prm->inject_species != 1, inj_e = prm->inject_species != 2;
    double *gp = malloc(sizeof(double) * nb * 9);
    if (!gp) return -1;
    double *ge = gp + nb, *src_p = gp + 2 * nb, *src_e = gp + 3 * nb;
    double *dlt_p = gp + 4 * nb, *dlt_e = gp + 5 * nb, *ad_p = gp + 6 * nb, *ad_e = gp + 7 * nb;
    double *scratch = gp + 8 * nb;
    dsa_grid_p(p_p, nb, prm->pmin_dsa_p_log10, gp);
    dsa_grid_p(p_e, nb, prm->pmin_dsa_e_log10, ge);
    const double mr = DSA_MP_G / DSA_ME_G;
    int count = 0;

    for (int t = 0; t < ntracer; t++) {
        double mach, temp, rho1, u1;
        if (!resolve_input(prm, sh, t, density_unit, &mach, &temp, &rho1, &u1)) continue;
        const double ratio = compression_ratio(mach, prm->gamma_gas);
        if (!(ratio > 0.0) || !isfinite(ratio)) continue;
        const double rho2 = ratio * rho1, u2 = u1 / ratio;
        const double q = slope_d3p(mach, prm->gamma_gas);
        if (!(q > 0.0) || !isfinite(q)) continue;
        const double pmin_p = injection_momentum(temp, prm->chi_p, DSA_MP_G);
        const double pmin_e = injection_momentum(temp, chi_e, DSA_ME_G);
        if (!(pmin_p > 0.0) || !isfinite(pmin_p) || !(pmin_e > 0.0) || !isfinite(pmin_e)) continue;

        /* fresh protons: dsa_build_proton_spectrum (the shock state fields
         * are already positive here) */
        int fresh_p = 0, fresh_e = 0;
        double A_p = 0.0;
        memset(src_p, 0, sizeof(double) * nb);
        memset(src_e, 0, sizeof(double) * nb);
        {
            const double eta = dsa_eta(mach, prm->eta_model_initial);
            if (mach > 1.0 && prm->gamma_gas > 1.0 && prm->chi_p > 0.0 && prm->pmax_p_mc > 0.0 &&
                eta > 0.0 && pmin_p < prm->pmax_p_mc) {
                const double unit = proton_edens_unit(pmin_p, q, prm->pmax_p_mc, 4000);
                if (unit > 0.0 && rho1 > 0.0 && u1 > 0.0 && u2 > 0.0)
                    A_p = eta * (0.5 * rho1 * u1 * u1 * u1) / u2 / unit;
                if (A_p > 0.0) {
                    fresh_p = 1;
                    for (int j = 0; j < nb; j++) src_p[j] = source_dp(A_p, pmin_p, q, prm->pmax_p_mc, gp[j]);
                }
            }
        }
        /* suprathermal electrons normalised to the protons at P = p_inj,p m_p c */
        if (fresh_p && inj_e && prm->pmax_e_mc > 0.0 && chi_e > 0.0 && pmin_e < prm->pmax_e_mc &&
            prm->k_ep > 0.0) {
            const double sp = spectrum_shape(pmin_p, pmin_p, q, prm->pmax_p_mc);
            const double se = spectrum_shape(mr * pmin_p, pmin_e, q, prm->pmax_e_mc);
            double A_e = 0.0;
            if (sp > 0.0 && se > 0.0) A_e = prm->k_ep * (1.0 / (mr * mr * mr)) * A_p * sp / se;
            if (A_e > 0.0) {
                fresh_e = 1;
                for (int j = 0; j < nb; j++) src_e[j] = source_dp(A_e, pmin_e, q, prm->pmax_e_mc, ge[j]);
            }
        }

        const double mass_g = mass_msun[t] * DSA_MSUN;
        const double vup = mass_g / rho1, vdown = mass_g / rho2;
        if (!(vup > 0.0) || !isfinite(vup) || !(vdown > 0.0) || !isfinite(vdown)) continue;
        const double *Np = crp + (size_t)t * nb, *Ne = cre + (size_t)t * nb;

        double scale = 0.0, energy = 0.0;
        memset(dlt_p, 0, sizeof(double) * nb);
        memset(dlt_e, 0, sizeof(double) * nb);
        if (reacc_mode == OR_REACC_POSITIVE) {
            double xcr = 0.0;
            const double ecr = edens_from_state(p_p, dp_p, Np, nb, vdown, prm->xcr_pmin_pmc, 0);
            const double pth = rho1 * DSA_KB_CGS * temp / (prm->mu_mol * DSA_MP_G);
            if (pth > 0.0 && isfinite(ecr / 3.0) && isfinite(pth) && ecr / 3.0 > 0.0) xcr = (ecr / 3.0) / pth;
            const double eta_p = dsa_eta(mach, prm->eta_model_initial);
            double eta_int;
            {
                const double ei = dsa_eta(mach, prm->eta_model_initial);
                const double er = dsa_eta(mach, prm->eta_model_reacc);
                const int valid = prm->eta_model_initial >= 0 && prm->eta_model_initial < 8 &&
                                  prm->eta_model_reacc >= 0 && prm->eta_model_reacc < 8;
                const double x0 = valid ? kModels[prm->eta_model_reacc].xcr0 : 0.0;
                if (!valid) {
                    eta_int = 0.0;
                } else if (x0 <= 0.0) {
                    eta_int = ei;
                } else {
                    double wgt = xcr / x0;
                    if (wgt < 0.0) wgt = 0.0;
                    if (wgt > 1.0) wgt = 1.0;
                    eta_int = (1.0 - wgt) * ei + wgt * er;
                }
            }
            double extra = eta_int - eta_p;
            if (extra < 0.0 || !isfinite(extra)) extra = 0.0;
            const double budget = extra * 0.5 * mass_g * u1 * u1;
            if (budget > 0.0) {
                const double ep = reacc_positive(p_p, dp_p, Np, nb, vdown, q, pmin_p, dlt_p, 0);
                const double ee = reacc_positive(p_e, dp_e, Ne, nb, vdown, q, pmin_e, dlt_e, 1);
                energy = (ep + ee) * vdown;
                if (energy > 0.0 && isfinite(energy)) {
                    scale = (energy > budget) ? budget / energy : 1.0;
                } else {
                    memset(dlt_p, 0, sizeof(double) * nb);
                    memset(dlt_e, 0, sizeof(double) * nb);
                }
            }
        } else if (reacc_mode == OR_REACC_DRURY83) {
            reacc_convolution(p_p, dp_p, Np, nb, vup, vdown, q, pmin_p, dlt_p, 0);
            reacc_convolution(p_e, dp_e, Ne, nb, vup, vdown, q, pmin_e, dlt_e, 1);
            const double cp = delta_edens(p_p, dp_p, dlt_p, nb, pmin_p, 0);
            const double ce = delta_edens(p_e, dp_e, dlt_e, nb, pmin_e, 1);
            energy = (cp + ce) * vdown;
            scale = 1.0;
            if (prm->reacc_eta_cap > 0.0 && isfinite(prm->reacc_eta_cap)) {
                const double budget = prm->reacc_eta_cap * 0.5 * mass_g * u1 * u1;
                const double ap = reacc_adiabatic(p_p, dp_p, Np, nb, vup, vdown, ratio, pmin_p, ad_p, scratch, 0);
                const double ae = reacc_adiabatic(p_e, dp_e, Ne, nb, vup, vdown, ratio, pmin_e, ad_e, scratch, 1);
                const double nonad = (cp + ce - ap - ae) * vdown;
                if (nonad > 0.0 && isfinite(nonad) && budget > 0.0 && isfinite(budget)) {
                    if (nonad > budget) scale = budget / nonad;
                    for (int j = 0; j < nb; j++) dlt_p[j] = ad_p[j] + scale * (dlt_p[j] - ad_p[j]);
                    for (int j = 0; j < nb; j++) dlt_e[j] = ad_e[j] + scale * (dlt_e[j] - ad_e[j]);
                    energy = (ap + ae + scale * (cp + ce - ap - ae)) * vdown;
                }
            }
            if (dis) dis[t] = 1;
        }

        int applied = 0;
        double *Op = (mode == OR_DSA_STATE) ? crp + (size_t)t * nb : qpi + (size_t)t * nb;
        double *Oe = (mode == OR_DSA_STATE) ? cre + (size_t)t * nb : qepri + (size_t)t * nb;
        const double inv_dt = (mode == OR_DSA_SOURCE) ? 1.0 / dt_gyr : 1.0;
        if (inj_p && fresh_p) {
            for (int j = 0; j < nb; j++)
                Op[j] += (mode == OR_DSA_STATE) ? src_p[j] * vdown : src_p[j] * vdown * inv_dt;
            applied = 1;
        }
        if (inj_e && fresh_p && fresh_e) {
            for (int j = 0; j < nb; j++)
                Oe[j] += (mode == OR_DSA_STATE) ? src_e[j] * vdown : src_e[j] * vdown * inv_dt;
            applied = 1;
        }
        if (reacc_mode == OR_REACC_POSITIVE || reacc_mode == OR_REACC_DRURY83) {
            const double s = (reacc_mode == OR_REACC_DRURY83) ? 1.0 : scale;
            for (int j = 0; j < nb; j++)
                Op[j] += (mode == OR_DSA_STATE) ? dlt_p[j] * vdown * s : dlt_p[j] * vdown * s * inv_dt;
            for (int j = 0; j < nb; j++)
                Oe[j] += (mode == OR_DSA_STATE) ? dlt_e[j] * vdown * s : dlt_e[j] * vdown * s * inv_dt;
            if (scale > 0.0 && isfinite(energy) && fabs(energy) > 0.0) applied = 1;
        }
        count += applied;
    }
    free(gp);
    if (ninjected) *ninjected = count;
    return 0;
}
