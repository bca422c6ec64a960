/*
 * ref_driver.c -- checker harness around the reference CPU implementation.
 *
 * Test infrastructure only.  This file is compiled together with the
 * reference's own CPU sources (see oracle/Makefile) into
 * oracle/_ref/libcroma_ref_np<N>.so.  It drives the reference's public CPU
 * functions through the same per-snapshot sequence as the reference
 * snapshot driver (include/tracer_fp_solve.inc):
 *
 *   1. IC-cooling rows for z and z_next
 *        tracer_fp_prepare_ic_cooling_snapshot  (src/tracer_fp_synch.c:242-294)
 *   2. endpoint loss prepass and N_subloop estimate
 *        tracer_fp_prepare_nsub_loss_endpoints  (src/tracer_fp_nsub.c:242-282)
 *        tracer_fp_compute_nsubsteps_from_endpoints (src/tracer_fp_nsub.c:217-240)
 *        (called as in include/tracer_fp_solve.inc:439-465)
 *   3. bucket build
 *        tracer_bucket_build_snapshot           (src/tracer_fp_bucket.c:208-262)
 *   4. CPU evolve with thread-local buckets
 *        tracer_fp_batch_execute_parallel       (src/tracer_fp_batch.c:829-1126)
 *        (called as in include/tracer_fp_solve.inc:618-673)
 *
 * plus direct entry points to single pieces (one segment evolve, one IC
 * row, coefficient batches, the secondary kernel) for fine-grained checks.
 * Backgrounds are passed as one field-major block [CROMA_BG_NFIELD][ntracer]
 * in the order n_gas, kbt, b_field, divv_gyr, l_turb_mpc, dv_imc, cs,
 * beta_pl.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "FP_Coef.h"
#include "fp_shared_core.h"
#include "tracer_fp.h"
#include "tracer_fp_batch.h"
#include "tracer_fp_bucket.h"
#include "tracer_fp_coef.h"
#include "tracer_fp_nsub.h"
#include "tracer_fp_synch.h"
#include "tracer_fp_setup.h"

enum {
    BG_NGAS = 0, BG_KBT, BG_BFIELD, BG_DIVV, BG_LTURB, BG_DV, BG_CS, BG_BETA,
    CROMA_BG_NFIELD
};

typedef struct {
    double pmin, pmax, pemin, pemax;
    int dpp_model;                 /* FP_MOMENTUMDIFF_MODEL_* */
    int ttd_tacc_model;            /* 0 spect, 1 brunetti16 */
    double t_acc_direct_gyr;
    double mach_limit;
    double psi;
    double eta_dpp_cap;
    double nsub_safety;
    int nsub_max;
    int coeff_interp_min_steps;
    int coeff_interp_max_segments;
    int reacc_window_mode;
    double f_eddy;
    double t_off_gyr;
    double t_acc_off_gyr;
    int nthreads;
} RefConfig;

static CRspectrum g_crp, g_cre;
static double g_beta_p[np];
static double g_gamma2e[npe];
static double g_fqe[(size_t)np * (size_t)npe];
static int g_np_min_qe[npe];
static int g_ready = 0;

int ref_np(void) { return np; }
int ref_npe(void) { return npe; }

int ref_configure(const RefConfig *cfg)
{
    if (cfg == 0) return -1;
    pmin = cfg->pmin;
    pmax = cfg->pmax;
    pemin = cfg->pemin;
    pemax = cfg->pemax;
    switch (cfg->dpp_model) {
    case FP_MOMENTUMDIFF_MODEL_ASA: strcpy(dpp_mode_spec, "asa"); break;
    case FP_MOMENTUMDIFF_MODEL_TTD: strcpy(dpp_mode_spec, "ttd"); break;
    case FP_MOMENTUMDIFF_MODEL_DIRECT_TACC: strcpy(dpp_mode_spec, "direct_tacc"); break;
    default: strcpy(dpp_mode_spec, "off"); break;
    }
    ttd_tacc_model = cfg->ttd_tacc_model;
    t_acc_direct_gyr = cfg->t_acc_direct_gyr;
    mach_limit = cfg->mach_limit;
    psi = cfg->psi;
    eta_dpp_cap = cfg->eta_dpp_cap;
    tracer_nsub_safety = cfg->nsub_safety;
    tracer_nsub_max = cfg->nsub_max;
    coeff_interp_min_steps = cfg->coeff_interp_min_steps;
    coeff_interp_max_segments = cfg->coeff_interp_max_segments;
    reacc_window_mode = cfg->reacc_window_mode;
    f_eddy = cfg->f_eddy;
    t_off_gyr = cfg->t_off_gyr;
    t_acc_off_gyr = cfg->t_acc_off_gyr;
#ifdef _OPENMP
    if (cfg->nthreads > 0) omp_set_num_threads(cfg->nthreads);
#endif
    memset(&g_crp, 0, sizeof(g_crp));
    memset(&g_cre, 0, sizeof(g_cre));
    momentum_bin(&g_crp, &g_cre, g_beta_p, g_gamma2e);
    momentumdiff_prepare_grid_cache(&g_crp, &g_cre);
    prepare_secondary_kernel_flat(&g_crp, &g_cre, g_beta_p, g_fqe, g_np_min_qe);
    g_ready = 1;
    return 0;
}

int ref_threads(void) { return tracer_fp_cpu_threads(); }

/* grid_out: [p(np), dp(np), E(np), pm1, pp1] for species 0 = proton,
 * [p(npe), dp(npe), E(npe), pm1, pp1] for species 1 = electron. */
int ref_get_grid(int species, double *grid_out)
{
    const CRspectrum *s = (species == 0) ? &g_crp : &g_cre;
    const int n = (species == 0) ? np : npe;
    if (!g_ready || grid_out == 0) return -1;
    memcpy(grid_out, s->p, (size_t)n * sizeof(double));
    memcpy(grid_out + n, s->dp, (size_t)n * sizeof(double));
    memcpy(grid_out + 2 * n, s->E, (size_t)n * sizeof(double));
    grid_out[3 * n] = s->pm1;
    grid_out[3 * n + 1] = s->pp1;
    return 0;
}

int ref_get_beta_p(double *out)
{
    if (!g_ready || out == 0) return -1;
    memcpy(out, g_beta_p, sizeof(g_beta_p));
    return 0;
}

/* Grid cache as used by the loss/Dpp code: sigma_pp, sigmoid_pp, j_pp. */
int ref_get_pp_cache(double *sigma_pp, double *sigmoid_pp, int *j_pp)
{
    if (!g_ready) return -1;
    if (sigma_pp) memcpy(sigma_pp, momentumdiff_crp_sigma_pp_cache(&g_crp), np * sizeof(double));
    if (sigmoid_pp) memcpy(sigmoid_pp, momentumdiff_crp_sigmoid_pp_cache(&g_crp), np * sizeof(double));
    if (j_pp) *j_pp = momentumdiff_crp_j_pp_cache(&g_crp);
    return 0;
}

int ref_get_secondary_kernel(double *fqe_flat, int *np_min_qe)
{
    if (!g_ready) return -1;
    if (fqe_flat) memcpy(fqe_flat, g_fqe, sizeof(g_fqe));
    if (np_min_qe) memcpy(np_min_qe, g_np_min_qe, sizeof(g_np_min_qe));
    return 0;
}

int ref_ic_row(double z, double *row, double *m1, double *p1)
{
    if (!g_ready) return -1;
    return prepare_ic_cooling_row(z, &g_cre, row, m1, p1);
}

int ref_nsub(int ntracer, double dt_snap, const double *bg, const double *rad_ic_row,
             int *nsub, int *target, int *non, unsigned char *capped)
{
    double *radic, *lo_p, *hi_p, *lo_e, *hi_e;
    int itr, je, ierr, maxn = 0, ncap = 0, maxraw = 0;
    if (!g_ready || ntracer <= 0) return -1;
    radic = (double *)malloc((size_t)npe * (size_t)ntracer * sizeof(double));
    lo_p = (double *)malloc((size_t)ntracer * 4 * sizeof(double));
    if (radic == 0 || lo_p == 0) { free(radic); free(lo_p); return -3; }
    hi_p = lo_p + ntracer; lo_e = hi_p + ntracer; hi_e = lo_e + ntracer;
    for (je = 0; je < npe; je++)
        for (itr = 0; itr < ntracer; itr++)
            radic[(size_t)je * ntracer + itr] = rad_ic_row[je];
    ierr = tracer_fp_prepare_nsub_loss_endpoints(
        ntracer, &g_crp, &g_cre,
        bg + (size_t)BG_NGAS * ntracer, bg + (size_t)BG_KBT * ntracer,
        bg + (size_t)BG_BFIELD * ntracer, bg + (size_t)BG_DIVV * ntracer,
        radic, lo_p, hi_p, lo_e, hi_e);
    if (ierr == 0) {
        ierr = tracer_fp_compute_nsubsteps_from_endpoints(
            ntracer, dt_snap, &g_crp, &g_cre, lo_p, hi_p, lo_e, hi_e,
            bg + (size_t)BG_LTURB * ntracer, bg + (size_t)BG_DV * ntracer,
            nsub, target, non, capped, &maxn, &ncap, &maxraw);
    }
    free(radic);
    free(lo_p);
    return ierr;
}

int ref_buckets(int ntracer, const int *nsub, const int *non,
                int *bucket_ids, int *indices, int *steps, int *onsteps,
                int *offsets, int *counts, int *nbuckets_out)
{
    TracerStep step;
    TracerBucket bucket;
    int ierr, nb = 0;
    memset(&step, 0, sizeof(step));
    memset(&bucket, 0, sizeof(bucket));
    step.nsubsteps = (int *)nsub;
    step.n_onsteps = (int *)non;
    if (tracer_bucket_alloc(&bucket, ntracer) != 0) { tracer_bucket_release(&bucket); return -3; }
    ierr = tracer_bucket_build_snapshot(&step, ntracer, &bucket, &nb);
    if (ierr == 0) {
        memcpy(bucket_ids, bucket.bucket_ids, (size_t)ntracer * sizeof(int));
        memcpy(indices, bucket.indices, (size_t)ntracer * sizeof(int));
        memcpy(steps, bucket.steps, (size_t)nb * sizeof(int));
        memcpy(onsteps, bucket.onsteps, (size_t)nb * sizeof(int));
        memcpy(offsets, bucket.member_offsets, (size_t)nb * sizeof(int));
        memcpy(counts, bucket.member_counts, (size_t)nb * sizeof(int));
        *nbuckets_out = nb;
    }
    tracer_bucket_release(&bucket);
    return ierr;
}

int ref_coeff_segments(int nsub, int allow_interp)
{
    return tracer_fp_choose_coeff_interp_segments(nsub, allow_interp);
}

/*
 * One coefficient batch + one segment of sub-steps for ncell tracers:
 * tracer_fp_cpu_evolve (src/tracer_fp_cpu.c:88-196).  bg is field-major
 * [8][ncell]; rad_ic is momentum-major [npe][ncell].  States are cell-major
 * and updated in place.
 */
int ref_evolve_segment(int ncell, int nstep, double dt,
                       int use_windowed_reacc, int on_start, int on_end,
                       const double *bg, const double *rad_ic,
                       const double *rad_ic_m1, const double *rad_ic_p1,
                       const double *qpi, const double *qepri,
                       const double *mass, const unsigned char *disable_adiabatic,
                       double *crp_state, double *cre_state)
{
    TracerFpGpuTimes times;
    TracerFpCpuWs ws;
    int ierr;
    if (!g_ready) return -1;
    memset(&times, 0, sizeof(times));
    memset(&ws, 0, sizeof(ws));
    ierr = tracer_fp_cpu_evolve(ncell, nstep, dt, use_windowed_reacc, on_start, on_end,
                                &g_crp, &g_cre,
                                bg + (size_t)BG_NGAS * ncell, bg + (size_t)BG_KBT * ncell,
                                bg + (size_t)BG_BFIELD * ncell, bg + (size_t)BG_DIVV * ncell,
                                bg + (size_t)BG_LTURB * ncell, bg + (size_t)BG_DV * ncell,
                                bg + (size_t)BG_CS * ncell, bg + (size_t)BG_BETA * ncell,
                                rad_ic, rad_ic_m1, rad_ic_p1, qpi, qepri,
                                g_fqe, g_np_min_qe, mass, disable_adiabatic,
                                crp_state, cre_state, &times, &ws);
    tracer_fp_cpu_ws_free(&ws);
    return ierr;
}

/*
 * Chang-Cooper tridiagonal rows for ncell tracers from one background, as
 * tracer_fp_prepare_coeff_batches builds them (src/tracer_fp_coef.c:218-359).
 * Outputs are cell-major [ncell][n]: on-set then off-set for each species.
 */
int ref_cc_coeffs(int ncell, double dt, const double *bg, const double *rad_ic,
                  const double *rad_ic_m1, const double *rad_ic_p1,
                  const double *mass, const unsigned char *disable_adiabatic,
                  const double *crp_state, const double *cre_state,
                  double *ccp_abc_on, double *cce_abc_on,
                  double *ccp_abc_off, double *cce_abc_off)
{
    TracerFpGpuTimes times;
    TracerFpCpuWs ws;
    double *qpi;
    size_t pn = (size_t)ncell * np, en = (size_t)ncell * npe;
    int ierr;
    if (!g_ready) return -1;
    memset(&times, 0, sizeof(times));
    memset(&ws, 0, sizeof(ws));
    qpi = (double *)calloc(pn + en, sizeof(double));
    if (qpi == 0) return -3;
    if (tracer_fp_cpu_ws_ensure(&ws, ncell) != 0) { free(qpi); return -3; }
    memset(ws.source.inje, 0, en * sizeof(double));
    ierr = tracer_fp_prepare_coeff_batches(ncell, dt, &g_crp, &g_cre,
                                           bg + (size_t)BG_NGAS * ncell, bg + (size_t)BG_KBT * ncell,
                                           bg + (size_t)BG_BFIELD * ncell, bg + (size_t)BG_DIVV * ncell,
                                           bg + (size_t)BG_LTURB * ncell, bg + (size_t)BG_DV * ncell,
                                           bg + (size_t)BG_CS * ncell, bg + (size_t)BG_BETA * ncell,
                                           rad_ic, rad_ic_m1, rad_ic_p1, qpi, qpi + pn,
                                           g_fqe, g_np_min_qe, mass, disable_adiabatic,
                                           crp_state, cre_state, &times, &ws);
    if (ierr == 0) {
        memcpy(ccp_abc_on, ws.cc.ccp_a, pn * sizeof(double));
        memcpy(ccp_abc_on + pn, ws.cc.ccp_b, pn * sizeof(double));
        memcpy(ccp_abc_on + 2 * pn, ws.cc.ccp_c, pn * sizeof(double));
        memcpy(cce_abc_on, ws.cc.cce_a, en * sizeof(double));
        memcpy(cce_abc_on + en, ws.cc.cce_b, en * sizeof(double));
        memcpy(cce_abc_on + 2 * en, ws.cc.cce_c, en * sizeof(double));
        memcpy(ccp_abc_off, ws.cc.ccp_a_off, pn * sizeof(double));
        memcpy(ccp_abc_off + pn, ws.cc.ccp_b_off, pn * sizeof(double));
        memcpy(ccp_abc_off + 2 * pn, ws.cc.ccp_c_off, pn * sizeof(double));
        memcpy(cce_abc_off, ws.cc.cce_a_off, en * sizeof(double));
        memcpy(cce_abc_off + en, ws.cc.cce_b_off, en * sizeof(double));
        memcpy(cce_abc_off + 2 * en, ws.cc.cce_c_off, en * sizeof(double));
    }
    tracer_fp_cpu_ws_free(&ws);
    free(qpi);
    return ierr;
}

/*
 * One full snapshot for ntracer tracers, following
 * include/tracer_fp_solve.inc (IC rows :104-115, nsub :439-465, buckets
 * :569-577, CPU thread-local evolve :618-673).  Returns the per-tracer
 * nsub / n_on and the bucket ids of the global bucket build.
 */
int ref_snapshot(int ntracer, const double *bg_curr, const double *bg_next,
                 double z_curr, double z_next, int allow_interp,
                 double dt_snap, double elapsed_gyr,
                 const double *qpi, const double *qepri, const double *mass,
                 const unsigned char *disable_adiabatic,
                 double *crp_state, double *cre_state,
                 int *nsub_out, int *non_out, int *bucket_ids_out, int *nbuckets_out)
{
    double *rad_ic_zero = 0, *rad_ic_m1 = 0, *rad_ic_p1 = 0;
    double rad_ic_row_next[npe];
    double m1_next = 0.0, p1_next = 0.0;
    double *lo_p = 0;
    int *nsub = 0, *target = 0, *non = 0, *base = 0, *cadence = 0;
    unsigned char *capped = 0, *dis = 0;
    int maxn = 0, ncap = 0, maxraw = 0, nb = 0, calls = 0, bmin = 0, bmax = 0;
    int ierr = -3;
    TracerStep step;
    TracerBucket bucket;
    TracerFpGpuTimes times;
    const double *bn = allow_interp ? bg_next : bg_curr;

    if (!g_ready || ntracer <= 0) return -1;
    memset(&step, 0, sizeof(step));
    memset(&bucket, 0, sizeof(bucket));
    memset(&times, 0, sizeof(times));

    rad_ic_zero = (double *)malloc((size_t)npe * (size_t)ntracer * sizeof(double));
    rad_ic_m1 = (double *)malloc((size_t)ntracer * sizeof(double));
    rad_ic_p1 = (double *)malloc((size_t)ntracer * sizeof(double));
    lo_p = (double *)malloc((size_t)ntracer * 4 * sizeof(double));
    nsub = (int *)calloc((size_t)ntracer, sizeof(int));
    target = (int *)calloc((size_t)ntracer, sizeof(int));
    non = (int *)calloc((size_t)ntracer, sizeof(int));
    base = (int *)calloc((size_t)ntracer, sizeof(int));
    cadence = (int *)calloc((size_t)ntracer, sizeof(int));
    capped = (unsigned char *)calloc((size_t)ntracer, 1);
    dis = (unsigned char *)calloc((size_t)ntracer, 1);
    if (!rad_ic_zero || !rad_ic_m1 || !rad_ic_p1 || !lo_p || !nsub || !target ||
        !non || !base || !cadence || !capped || !dis) goto done;
    if (disable_adiabatic) memcpy(dis, disable_adiabatic, (size_t)ntracer);

    ierr = tracer_fp_prepare_ic_cooling_snapshot(ntracer, allow_interp, z_curr,
                                                 allow_interp ? z_next : z_curr, &g_cre,
                                                 rad_ic_zero, rad_ic_m1, rad_ic_p1,
                                                 rad_ic_row_next, &m1_next, &p1_next);
    if (ierr != 0) goto done;

    ierr = tracer_fp_prepare_nsub_loss_endpoints(
        ntracer, &g_crp, &g_cre,
        bg_curr + (size_t)BG_NGAS * ntracer, bg_curr + (size_t)BG_KBT * ntracer,
        bg_curr + (size_t)BG_BFIELD * ntracer, bg_curr + (size_t)BG_DIVV * ntracer,
        rad_ic_zero, lo_p, lo_p + ntracer, lo_p + 2 * (size_t)ntracer, lo_p + 3 * (size_t)ntracer);
    if (ierr != 0) goto done;
    ierr = tracer_fp_compute_nsubsteps_from_endpoints(
        ntracer, dt_snap, &g_crp, &g_cre,
        lo_p, lo_p + ntracer, lo_p + 2 * (size_t)ntracer, lo_p + 3 * (size_t)ntracer,
        bg_curr + (size_t)BG_LTURB * ntracer, bg_curr + (size_t)BG_DV * ntracer,
        nsub, target, non, capped, &maxn, &ncap, &maxraw);
    if (ierr != 0) goto done;
    for (int i = 0; i < ntracer; i++) { base[i] = nsub[i]; cadence[i] = 1; }

    step.nsubsteps = nsub;
    step.n_onsteps = non;
    if (tracer_bucket_alloc(&bucket, ntracer) != 0) { ierr = -3; goto done; }
    ierr = tracer_bucket_build_snapshot(&step, ntracer, &bucket, &nb);
    if (ierr != 0) goto done;

    ierr = tracer_fp_batch_execute_parallel(
        ntracer, nsub, non, base, cadence, TRACER_FP_INTEGRATION_QUANTIZED,
        allow_interp, elapsed_gyr, dt_snap, z_curr, allow_interp ? z_next : z_curr,
        t_acc_direct_gyr, &g_crp, &g_cre,
        bg_curr + (size_t)BG_NGAS * ntracer, bg_curr + (size_t)BG_KBT * ntracer,
        bg_curr + (size_t)BG_BFIELD * ntracer, bg_curr + (size_t)BG_DIVV * ntracer,
        bg_curr + (size_t)BG_LTURB * ntracer, bg_curr + (size_t)BG_DV * ntracer,
        bg_curr + (size_t)BG_CS * ntracer, bg_curr + (size_t)BG_BETA * ntracer,
        rad_ic_zero, rad_ic_m1, rad_ic_p1,
        bn + (size_t)BG_NGAS * ntracer, bn + (size_t)BG_KBT * ntracer,
        bn + (size_t)BG_BFIELD * ntracer, bn + (size_t)BG_DIVV * ntracer,
        bn + (size_t)BG_LTURB * ntracer, bn + (size_t)BG_DV * ntracer,
        bn + (size_t)BG_CS * ntracer, bn + (size_t)BG_BETA * ntracer,
        rad_ic_row_next, m1_next, p1_next,
        qpi, qepri, g_fqe, g_np_min_qe, mass, dis,
        crp_state, cre_state, &times, &calls, &bmin, &bmax);
    if (ierr != 0) goto done;

    if (nsub_out) memcpy(nsub_out, nsub, (size_t)ntracer * sizeof(int));
    if (non_out) memcpy(non_out, non, (size_t)ntracer * sizeof(int));
    if (bucket_ids_out) memcpy(bucket_ids_out, bucket.bucket_ids, (size_t)ntracer * sizeof(int));
    if (nbuckets_out) *nbuckets_out = nb;

done:
    tracer_bucket_release(&bucket);
    free(rad_ic_zero); free(rad_ic_m1); free(rad_ic_p1); free(lo_p);
    free(nsub); free(target); free(non); free(base); free(cadence);
    free(capped); free(dis);
    return ierr;
}

/* ---- DSA injection through the reference's own snapshot routine ----
 * Sets the reference's DSA globals (src/params.c:96-113, mu_mol :127) from
 * prm, builds its DSA grid (dsa_init_grid, src/DSA_MODELS.c:1191) on the
 * configured FP grids and calls tracer_fp_apply_dsa_tracer_injection_snapshot
 * (src/tracer_fp_dsa.c:184) on cell-major state. */
#include "DSA_MODELS.h"
#include "tracer_fp_dsa.h"
#include "croma_oracle.h"

int ref_dsa_inject(const OrDsaParams *prm, const OrShockFields *sh, int ntracer,
                   const double *mass_msun, double density_unit, double dt_gyr, int mode,
                   int reacc_mode, double *crp, double *cre, double *qpi, double *qepri,
                   unsigned char *dis, int *ninjected)
{
    DSAGrid grid;
    TracerFpRawBackgroundSlot raw;
    int rc;
    if (!g_ready || !prm || !sh) return -1;
    DSAEtaModelInitial = (DSAModelID)prm->eta_model_initial;
    DSAEtaModelReacc = (DSAModelID)prm->eta_model_reacc;
    DSAChiP = prm->chi_p;
    DSAChiE = prm->chi_e;
    DSAKep = prm->k_ep;
    DSAPmaxPmc = prm->pmax_p_mc;
    DSAPmaxEmc = prm->pmax_e_mc;
    DSAMinMach = prm->min_mach;
    DSAGammaGas = prm->gamma_gas;
    DSAXcrPminPmc = prm->xcr_pmin_pmc;
    DSAReaccEtaCap = prm->reacc_eta_cap;
    DSAInjectSpecies = prm->inject_species;
    DSADebug = 0;
    mu_mol = prm->mu_mol;
    memset(&grid, 0, sizeof grid);
    if (!dsa_init_grid(&grid, &g_crp, &g_cre, prm->pmin_dsa_p_log10, prm->pmin_dsa_e_log10)) return -1;
    memset(&raw, 0, sizeof raw);
    raw.mach = (double *)sh->mach;
    raw.prestemp = (double *)sh->prestemp;
    raw.presden = (double *)sh->presden;
    raw.pre_density_cgs = (double *)sh->pre_density_cgs;
    raw.upstream_speed_cgs = (double *)sh->upstream_speed_cgs;
    raw.shock_side_code = (double *)sh->shock_side_code;
    raw.dsa_trigger = (double *)sh->dsa_trigger;
    raw.dsa_mach = (double *)sh->dsa_mach;
    raw.dsa_pre_density = (double *)sh->dsa_pre_density;
    raw.dsa_kinetic_energy_flux_cgs = (double *)sh->dsa_flux_cgs;
    raw.has_shock = 1;
    raw.has_dsa = sh->has_dsa;
    rc = tracer_fp_apply_dsa_tracer_injection_snapshot(
        &raw, ntracer, NULL, mass_msun, density_unit, dt_gyr, (TracerDsaInjectionMode)mode,
        (TracerDsaReaccMode)reacc_mode, &g_crp, &g_cre, &grid, crp, cre, qpi, qepri, dis,
        1, 0, NULL, ninjected);
    dsa_free_grid(&grid);
    return rc;
}

/* IC emissivity through the reference: the kernel table of
 * prepare_ic_kernel_flat (src/fp_shared_core.c:1780-1807) for nbins bands over
 * [nu_min, nu_max] (log10 Hz) at redshift z, and prepare_ic_emission_batch
 * (src/fp_shared_core.c:2131-2164) on cell-major electron spectra. */
int ref_ic_emission(int ncell, int nbins, double z, double nu_min, double nu_max,
                    const double *cre, double *fic_out, double *eps_out)
{
    FpIcEmissionBatchInput in;
    if (!g_ready || ncell <= 0 || nbins <= 0 || !cre || !fic_out || !eps_out) return -1;
    prepare_ic_kernel_flat(&g_cre, nbins, nu_min, nu_max, z, fic_out);
    memset(&in, 0, sizeof in);
    in.ncell = ncell;
    in.nbins = nbins;
    in.z = z;
    in.nu_min = nu_min;
    in.nu_max = nu_max;
    in.cre_batch = cre;
    in.fic_flat = fic_out;
    return prepare_ic_emission_batch(&in, &g_cre, eps_out);
}

/* ---- synchrotron emission on caller tables -------------------------------
 * logy [nfreq][npe][ntheta] flat; the pointer views the reference expects
 * are built here.  ref_synch_pitch_table runs prepare_synch_pitch_kernel_table
 * (src/fp_shared_core.c:2008-2052); ref_synch_emission runs
 * prepare_synch_emission_cell_major (src/fp_shared_core.c:2070-2129) with the
 * table when one is given and through SYN_emissivity_from_arrays
 * (src/Synchrotron.c:62-103) otherwise, whose pitch loop runs over the
 * global tracer_synch_ntheta_pitch, set here to ntheta. */
static int synch_input(FpSynchEmissionBatchInput *in, int nfreq, int nx, int ntheta, int nlogb, double xmin,
                       double logb_min, double inv_dlogb, const double *fx, const double *logfx,
                       const double *logx, const double *logy, const double *w, double ****planes_out)
{
    double ***planes = (double ***)calloc((size_t)nfreq, sizeof(double **));
    double **rows = (double **)calloc((size_t)nfreq * (size_t)npe, sizeof(double *));
    int nf, je;
    if (!planes || !rows) { free(planes); free(rows); return -1; }
    for (nf = 0; nf < nfreq; nf++) {
        planes[nf] = rows + (size_t)nf * (size_t)npe;
        for (je = 0; je < npe; je++)
            planes[nf][je] = (double *)logy + ((size_t)nf * (size_t)npe + (size_t)je) * (size_t)ntheta;
    }
    memset(in, 0, sizeof *in);
    in->nfreq = nfreq;
    in->nx_tab = nx;
    in->ntheta_pitch = ntheta;
    in->nlogb = nlogb;
    in->xmin = xmin;
    in->logb_min = logb_min;
    in->inv_dlogb = inv_dlogb;
    in->fx_tab = fx;
    in->logfx_tab = logfx;
    in->logx_tab = logx;
    in->logy = planes;
    in->pitch_weight = w;
    *planes_out = planes;
    return 0;
}

static void synch_input_free(double ***planes)
{
    if (!planes) return;
    free(planes[0]);
    free(planes);
}

int ref_synch_pitch_table(int nfreq, int nx, int ntheta, int nlogb, double xmin, double logb_min,
                          double inv_dlogb, const double *fx, const double *logfx, const double *logx,
                          const double *logy, const double *w, double *table_out)
{
    FpSynchEmissionBatchInput in;
    double ***planes = 0;
    int rc;
    if (synch_input(&in, nfreq, nx, ntheta, nlogb, xmin, logb_min, inv_dlogb, fx, logfx, logx, logy, w,
                    &planes) != 0)
        return -1;
    rc = prepare_synch_pitch_kernel_table(&in, table_out);
    synch_input_free(planes);
    return rc;
}

int ref_synch_emission(int ncell, int nfreq, int nx, int ntheta, int nlogb, double xmin, double logb_min,
                       double inv_dlogb, const double *fx, const double *logfx, const double *logx,
                       const double *logy, const double *w, const double *table, const double *b_dyn,
                       const double *logb, const double *cre, double *eps_out)
{
    FpSynchEmissionBatchInput in;
    double ***planes = 0;
    double *dummy;
    int rc;
    if (!g_ready) return -1;
    if (synch_input(&in, nfreq, nx, ntheta, nlogb, xmin, logb_min, inv_dlogb, fx, logfx, logx, logy, w,
                    &planes) != 0)
        return -1;
    /* fields the routine checks for but this branch does not read */
    dummy = (double *)calloc((size_t)(npe > ntheta ? npe : ntheta) + (size_t)nfreq, sizeof(double));
    in.ncell = ncell;
    in.pitch_kernel_table = table;
    in.b_dyn = b_dyn;
    in.logb = logb;
    in.cre_batch = cre;
    in.gamma2e = dummy;
    in.theta = dummy;
    in.dtheta = dummy;
    in.nus = dummy;
    tracer_synch_ntheta_pitch = ntheta;
    rc = dummy ? prepare_synch_emission_cell_major(&in, &g_cre, eps_out) : -1;
    free(dummy);
    synch_input_free(planes);
    return rc;
}

/* ---- emission kernel tables and full emission through the reference ----
 * ref_gamma_kernel_table / ref_nu_kernel_table / ref_ic_kernel_table run
 * prepare_{gamma,neutrino,ic}_kernel_flat (src/fp_shared_core.c:1724-1807);
 * ref_hadronic_emission runs prepare_{gamma,neutrino}_emission_cell_major
 * (:2166-2243) with the grid's beta_p.  ref_synch_run builds the reference's
 * SynchData with tracer_fp_synch_data_init_tables (src/tracer_fp_synch.c:87-121;
 * its F(x) column comes from oracle/synch_fx.c through the GSL stand-in), the
 * pitch-kernel table of tracer_fp_refresh_synch_kernel_table (:175-240, fixed
 * log-B range) and prepare_synch_emission_cell_major (:2070-2129) on b_dyn,
 * as include/tracer_fp_solve.inc:117-186 does; every table is returned. */
int ref_gamma_kernel_table(int nbins, double emin, double emax, double *out)
{
    if (!g_ready || nbins <= 0 || !out) return -1;
    prepare_gamma_kernel_flat(&g_crp, nbins, emin, emax, out);
    return 0;
}

int ref_nu_kernel_table(int nbins, double emin, double emax, double *out)
{
    if (!g_ready || nbins <= 0 || !out) return -1;
    prepare_neutrino_kernel_flat(&g_crp, nbins, emin, emax, out);
    return 0;
}

int ref_ic_kernel_table(int nbins, double nu_min, double nu_max, double z, double *out)
{
    if (!g_ready || nbins <= 0 || !out) return -1;
    prepare_ic_kernel_flat(&g_cre, nbins, nu_min, nu_max, z, out);
    return 0;
}

/* kind 0 gamma, 1 neutrino */
int ref_hadronic_emission(int kind, int ncell, int nbins, double emin, double emax, const double *n_gas,
                          const double *crp, const double *kern, double *eps_out)
{
    if (!g_ready || ncell <= 0 || nbins <= 0) return -1;
    if (kind == 0) {
        FpGammaEmissionBatchInput in;
        memset(&in, 0, sizeof in);
        in.ncell = ncell; in.nbins = nbins; in.egamma_min = emin; in.egamma_max = emax;
        in.n_gas = n_gas; in.crp_batch = crp; in.beta_p = g_beta_p; in.fga_flat = kern;
        return prepare_gamma_emission_cell_major(&in, &g_crp, eps_out);
    } else {
        FpNeutrinoEmissionBatchInput in;
        memset(&in, 0, sizeof in);
        in.ncell = ncell; in.nbins = nbins; in.enu_min = emin; in.enu_max = emax;
        in.n_gas = n_gas; in.crp_batch = crp; in.beta_p = g_beta_p; in.fnu_flat = kern;
        return prepare_neutrino_emission_cell_major(&in, &g_crp, eps_out);
    }
}

/* Outputs (any may be NULL): logx/logfx/fx [2750], theta/w [ntheta],
 * nus [nfreq], logy [nfreq][npe][ntheta], table [nlogb][nfreq][npe],
 * eps [ncell][nfreq] (ncell > 0 with b_field and cre). */
int ref_synch_run(int nfreq, double nu_min, double nu_max, int ntheta, int nlogb, double logb_min,
                  double logb_max, int ncell, const double *b_field, const double *cre,
                  double *logx, double *logfx, double *fx, double *theta, double *w, double *nus,
                  double *logy, double *table, double *eps)
{
    SynchData sd;
    int rc = 0, nlogb_saved = 0;
    double *b_dyn = 0, *lb = 0, lbmin = 0.0, lbmax = 0.0;
    int nout = 0;
    (void)nlogb_saved;
    if (!g_ready || nfreq <= 0 || ntheta <= 0) return -1;
    if (nlogb != TRACER_FP_SYNCH_LOGB_BINS) return -2;   /* the reference's table has a fixed plane count */
    nu_min_s = nu_min;
    nu_max_s = nu_max;
    tracer_synch_ntheta_pitch = ntheta;
    tracer_synch_logb_min = logb_min;
    tracer_synch_logb_max = logb_max;
    adaptive_synch_logb = 0;
    tracer_fp_synch_data_reset(&sd);
    if (tracer_fp_synch_data_alloc(&sd, nfreq) != 0 ||
        tracer_fp_synch_data_init_tables(&sd, nfreq, &g_cre) != 0) {
        tracer_fp_synch_data_release(&sd);
        return -1;
    }
    if (logx) memcpy(logx, sd.logx_tab, (size_t)sd.nx_tab * sizeof(double));
    if (logfx) memcpy(logfx, sd.logfx_tab, (size_t)sd.nx_tab * sizeof(double));
    if (fx) memcpy(fx, sd.fx_tab, (size_t)sd.nx_tab * sizeof(double));
    if (theta) memcpy(theta, sd.theta, (size_t)ntheta * sizeof(double));
    if (w) memcpy(w, sd.pitch_weight, (size_t)ntheta * sizeof(double));
    if (nus) memcpy(nus, sd.nus, (size_t)nfreq * sizeof(double));
    if (logy) memcpy(logy, sd.logy_storage, (size_t)nfreq * (size_t)npe * (size_t)ntheta * sizeof(double));
    if (tracer_fp_refresh_synch_kernel_table(&sd, nfreq, 0.0, 0.0, &sd.kernel_table) != 0) {
        tracer_fp_synch_data_release(&sd);
        return -1;
    }
    if (table) memcpy(table, sd.kernel_table, (size_t)nlogb * (size_t)nfreq * (size_t)npe * sizeof(double));
    if (ncell > 0 && b_field && cre && eps) {
        FpSynchEmissionBatchInput in;
        int i;
        b_dyn = (double *)malloc((size_t)ncell * sizeof(double));
        lb = (double *)malloc((size_t)ncell * sizeof(double));
        if (!b_dyn || !lb) { rc = -1; goto done; }
        for (i = 0; i < ncell; i++) b_dyn[i] = b_field[i];
        tracer_fp_logb_range_from_snapshot(ncell, b_dyn, lb, &lbmin, &lbmax, &nout);
        memset(&in, 0, sizeof in);
        in.ncell = ncell;
        in.nfreq = nfreq;
        in.nx_tab = sd.nx_tab;
        in.ntheta_pitch = sd.ntheta_pitch;
        in.nlogb = TRACER_FP_SYNCH_LOGB_BINS;
        in.xmin = sd.xmin;
        in.logb_min = sd.table_logb_min;
        in.inv_dlogb = (double)(TRACER_FP_SYNCH_LOGB_BINS - 1) / (sd.table_logb_max - sd.table_logb_min);
        in.fx_tab = sd.fx_tab;
        in.logfx_tab = sd.logfx_tab;
        in.logx_tab = sd.logx_tab;
        in.logy = sd.logy_planes;
        in.pitch_kernel_table = sd.kernel_table;
        in.b_dyn = b_dyn;
        in.logb = lb;
        in.cre_batch = cre;
        in.gamma2e = g_gamma2e;
        in.theta = sd.theta;
        in.dtheta = sd.dtheta;
        in.pitch_weight = sd.pitch_weight;
        in.nus = sd.nus;
        rc = prepare_synch_emission_cell_major(&in, &g_cre, eps);
    }
done:
    free(b_dyn);
    free(lb);
    tracer_fp_synch_data_release(&sd);
    return rc;
}

/* ---- output files and checkpoints (src/tracer_fp_output.c,
 * src/tracer_fp_restart.c) on caller arrays, for byte comparisons --------
 * Open writers live in a small table indexed by the returned handle. */
#include "tracer_fp_output.h"
#include "tracer_fp_restart.h"

#define REF_MAX_OUT 8
static TracerFpTileOutput g_tiles[REF_MAX_OUT];
static TracerFpMappedOutput g_maps[REF_MAX_OUT];
static int g_tile_used[REF_MAX_OUT], g_map_used[REF_MAX_OUT];

int ref_tile_open(const char *dir, const char *stem, int rank, long nslab, long nrow, long ncol, int resume)
{
    int h;
    for (h = 0; h < REF_MAX_OUT && g_tile_used[h]; h++) {}
    if (h == REF_MAX_OUT) return -1;
    if (tracer_fp_tile_open(&g_tiles[h], dir, stem, rank, (size_t)nslab, (size_t)nrow, (size_t)ncol, resume) != 0)
        return -1;
    g_tile_used[h] = 1;
    return h;
}

int ref_tile_write_cr(int h_e, int h_p, int nlocal, long slab, const double *cre, const double *crp,
                      const double *rho, const double *mass, int per_cc, int write_crp)
{
    if (h_e < 0 || h_e >= REF_MAX_OUT || !g_tile_used[h_e]) return -1;
    return tracer_fp_tile_write_cr(&g_tiles[h_e], h_p >= 0 ? &g_tiles[h_p] : 0, nlocal, (size_t)slab, cre, crp,
                                   rho, mass, per_cc, write_crp);
}

int ref_tile_write_emit(int h, int nlocal, long slab, int nbin, const double *eps, const double *rho,
                        const double *mass, int per_cc)
{
    if (h < 0 || h >= REF_MAX_OUT || !g_tile_used[h]) return -1;
    return tracer_fp_tile_write_emit(&g_tiles[h], nlocal, (size_t)slab, nbin, eps, rho, mass, per_cc);
}

int ref_tile_close(int h)
{
    if (h < 0 || h >= REF_MAX_OUT || !g_tile_used[h]) return -1;
    g_tile_used[h] = 0;
    return tracer_fp_tile_close(&g_tiles[h]);
}

int ref_map_open(const char *dir, const char *stem, int rank, int nrow, long ncol, int resume)
{
    int h;
    for (h = 0; h < REF_MAX_OUT && g_map_used[h]; h++) {}
    if (h == REF_MAX_OUT) return -1;
    if (tracer_fp_map_open(&g_maps[h], dir, stem, rank, nrow, (size_t)ncol, resume) != 0) return -1;
    g_map_used[h] = 1;
    return h;
}

int ref_write_cr_map(int h_e, int h_p, int nlocal, int slot, const double *cre, const double *crp,
                     const double *rho, const double *mass, int per_cc)
{
    if (h_e < 0 || h_e >= REF_MAX_OUT || !g_map_used[h_e]) return -1;
    return tracer_fp_write_cr_map(&g_maps[h_e], h_p >= 0 ? &g_maps[h_p] : 0, nlocal, slot, cre, crp, rho, mass,
                                  per_cc);
}

int ref_write_emit_map(int h, int nlocal, int snapshot_index, int nbin, const double *eps, const double *rho,
                       const double *mass, int per_cc)
{
    if (h < 0 || h >= REF_MAX_OUT || !g_map_used[h]) return -1;
    return tracer_fp_write_emit_map(&g_maps[h], nlocal, snapshot_index, nbin, eps, rho, mass, per_cc);
}

int ref_map_close(int h)
{
    if (h < 0 || h >= REF_MAX_OUT || !g_map_used[h]) return -1;
    g_map_used[h] = 0;
    return tracer_fp_map_close(&g_maps[h]);
}

/* tracer_fp_ckpt_write / tracer_fp_ckpt_read with the snapshot index range
 * globals nsnp_i / nsnp_f (params.c) set for the header. */
int ref_ckpt_write(const char *dir, int rank, int world, int ntracer, int ntracer_global, int nsnap, int nfreq,
                   int completed, long tracer_start, const int *ids, const double *crp, const double *cre,
                   int nsnp_i_value, int nsnp_f_value)
{
    TracerFpCkptWrite w;
    nsnp_i = nsnp_i_value;
    nsnp_f = nsnp_f_value;
    memset(&w, 0, sizeof w);
    w.checkpoint_dir = dir;
    w.mpi_rank = rank;
    w.world_size = world;
    w.ntracer = ntracer;
    w.ntracer_global = ntracer_global;
    w.nsnap = nsnap;
    w.nfreq = nfreq;
    w.completed_snapshot = completed;
    w.tracer_start = tracer_start;
    w.tracer_ids = ids;
    w.crp_state = crp;
    w.cre_state = cre;
    return tracer_fp_ckpt_write(&w);
}

int ref_ckpt_read(const char *dir, int rank, int world, int ntracer, int ntracer_global, int nsnap, int nfreq,
                  long tracer_start, const int *ids, double *crp, double *cre, int nsnp_i_value,
                  int nsnp_f_value, int *completed)
{
    TracerFpCkptRead r;
    nsnp_i = nsnp_i_value;
    nsnp_f = nsnp_f_value;
    memset(&r, 0, sizeof r);
    r.restart_dir = dir;
    r.mpi_rank = rank;
    r.world_size = world;
    r.ntracer = ntracer;
    r.ntracer_global = ntracer_global;
    r.nsnap = nsnap;
    r.nfreq = nfreq;
    r.tracer_start = tracer_start;
    r.tracer_ids = ids;
    r.crp_state = crp;
    r.cre_state = cre;
    r.completed_snapshot_out = completed;
    return tracer_fp_ckpt_read(&r);
}
