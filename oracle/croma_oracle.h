/*
 * croma_oracle.h -- CPU restatement of CROMA's per-tracer Fokker-Planck
 * update (kosukenishiwaki/croma-fp), used ONLY as the checker by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py.  Nothing in
 * the product links or calls it.
 *
 * Bin counts are a runtime argument here (np == npe == nb); in the
 * reference they are compile-time macros (include/params.h:22-27).
 * The restatement is pinned against the reference's own CPU code compiled
 * from its sources (oracle/_ref, see oracle/Makefile).
 */
#ifndef CROMA_ORACLE_H
#define CROMA_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Background field order of a field-major block [OR_BG_NFIELD][ntracer]. */
enum {
    OR_BG_NGAS = 0, OR_BG_KBT, OR_BG_BFIELD, OR_BG_DIVV,
    OR_BG_LTURB, OR_BG_DV, OR_BG_CS, OR_BG_BETA, OR_BG_NFIELD
};

/* FP_MOMENTUMDIFF_MODEL_* values of include/fp_shared_core.h:227-233. */
enum { OR_DPP_ASA = 1, OR_DPP_TTD = 2, OR_DPP_OFF = 3, OR_DPP_DIRECT = 4 };

typedef struct {
    int nb;                       /* bins per species, np == npe */
    double pmin, pmax;            /* log10 proton grid bounds (params.c pmin/pmax) */
    double pemin, pemax;          /* log10 electron grid bounds */
    int dpp_model;                /* OR_DPP_* */
    int ttd_tacc_model;           /* 0 spectral, 1 brunetti16 */
    double t_acc_direct_gyr;
    double mach_limit;
    double psi;
    double eta_dpp_cap;
    double nsub_safety;
    int nsub_max;
    int coeff_interp_min_steps;
    int coeff_interp_max_segments;
    int reacc_window_mode;        /* 0 always on, 1 centred */
    double f_eddy;
    double t_off_gyr;
    double t_acc_off_gyr;
} OrParams;

typedef struct OrCtx OrCtx;

OrCtx *or_create(const OrParams *par);
void or_destroy(OrCtx *ctx);

/* grid_out: p[nb], dp[nb], E[nb], pm1, pp1 (3*nb+2 doubles); species 0 = p, 1 = e */
int or_get_grid(const OrCtx *ctx, int species, double *grid_out);
int or_get_beta_p(const OrCtx *ctx, double *out);
int or_get_pp_cache(const OrCtx *ctx, double *sigma_pp, double *sigmoid_pp, int *j_pp);
int or_get_secondary_kernel(const OrCtx *ctx, double *fqe_flat, int *np_min_qe);

int or_ic_row(const OrCtx *ctx, double z, double *row, double *m1, double *p1);

int or_nsub(const OrCtx *ctx, int ntracer, double dt_snap, const double *bg,
            const double *rad_ic_row, int *nsub, int *target, int *non,
            unsigned char *capped);

int or_buckets(int ntracer, const int *nsub, const int *non, int *bucket_ids,
               int *indices, int *steps, int *onsteps, int *offsets,
               int *counts, int *nbuckets_out);

int or_coeff_segments(const OrCtx *ctx, int nsub, int allow_interp);

/* Chang-Cooper rows for one background of ncell tracers; outputs cell-major
 * [3][ncell][nb] (a, b, c) for each species and coefficient set. */
int or_cc_coeffs(const OrCtx *ctx, int ncell, double dt, const double *bg,
                 const double *rad_ic, const double *rad_ic_m1,
                 const double *rad_ic_p1, const double *mass,
                 const unsigned char *disable_adiabatic,
                 const double *crp_state, const double *cre_state,
                 double *ccp_on, double *cce_on, double *ccp_off, double *cce_off);

/* One segment for ncell tracers (tracer_fp_cpu_evolve semantics);
 * rad_ic is momentum-major [nb][ncell]. */
int or_evolve_segment(const OrCtx *ctx, int ncell, int nstep, double dt,
                      int use_windowed_reacc, int on_start, int on_end,
                      const double *bg, const double *rad_ic,
                      const double *rad_ic_m1, const double *rad_ic_p1,
                      const double *qpi, const double *qepri, const double *mass,
                      const unsigned char *disable_adiabatic,
                      double *crp_state, double *cre_state);

/* One full snapshot (IC rows, nsub, buckets, per-tracer evolve). */
int or_snapshot(const OrCtx *ctx, int ntracer, const double *bg_curr,
                const double *bg_next, double z_curr, double z_next,
                int allow_interp, double dt_snap, double elapsed_gyr,
                const double *qpi, const double *qepri, const double *mass,
                const unsigned char *disable_adiabatic,
                double *crp_state, double *cre_state,
                int *nsub_out, int *non_out, int *bucket_ids_out, int *nbuckets_out);

/* Same snapshot with the IC rows supplied by the caller (row_curr/row_next
 * are nb+2 doubles: row, m1, p1).  Used to isolate the evolve. */
int or_snapshot_with_ic(const OrCtx *ctx, int ntracer, const double *bg_curr,
                        const double *bg_next, const double *ic_curr,
                        const double *ic_next, int allow_interp, double dt_snap,
                        double elapsed_gyr, const double *qpi, const double *qepri,
                        const double *mass, const unsigned char *disable_adiabatic,
                        double *crp_state, double *cre_state,
                        int *nsub_out, int *non_out, int *bucket_ids_out,
                        int *nbuckets_out);

void or_set_threads(int n);

/* ---- DSA injection (croma_oracle_dsa.c) ---- */
enum { OR_DSA_OFF = 0, OR_DSA_STATE = 1, OR_DSA_SOURCE = 2 };          /* TracerDsaInjectionMode */
enum { OR_REACC_OFF = 0, OR_REACC_POSITIVE = 1, OR_REACC_DRURY83 = 2 }; /* TracerDsaReaccMode */

/* The DSA run parameters (src/params.c:96-113 and mu_mol, :127); model ids
 * follow DSAModelID: 0 KR07, 1 KR07r, 2 KR13, 3 KR13r, 4 CS14, 5 CS14r,
 * 6 Ryu19, 7 Ryu19r.  inject_species: 0 both, 1 electrons, 2 protons. */
typedef struct {
    int eta_model_initial, eta_model_reacc;
    double chi_p, chi_e, k_ep, pmax_p_mc, pmax_e_mc;
    double min_mach, gamma_gas, xcr_pmin_pmc, reacc_eta_cap, mu_mol;
    double pmin_dsa_p_log10, pmin_dsa_e_log10;   /* dsa_init_grid bounds */
    int inject_species;
} OrDsaParams;

/* Per-tracer shock fields [ntracer] (TracerFpRawBackgroundSlot,
 * include/tracer_fp_types.h:292-313); optional arrays may be NULL. */
typedef struct {
    const double *mach, *prestemp, *presden, *pre_density_cgs, *upstream_speed_cgs, *shock_side_code;
    const double *dsa_trigger, *dsa_mach, *dsa_pre_density, *dsa_flux_cgs;
    int has_dsa;
} OrShockFields;

/* tracer_fp_apply_dsa_tracer_injection_snapshot on cell-major state. */
int or_dsa_inject(const OrDsaParams *prm, int nb, const double *p_p, const double *dp_p,
                  const double *p_e, const double *dp_e, const OrShockFields *sh, int ntracer,
                  const double *mass_msun, double density_unit, double dt_gyr, int mode,
                  int reacc_mode, double *crp, double *cre, double *qpi, double *qepri,
                  unsigned char *dis, int *ninjected);

/* ---- background preparation (croma_oracle_background.c) ---- */
/* bg[8][n] from one snapshot's raw fields; -2 if a tracer has density <= 0. */
int or_background(int n, const double *temp_K, const double *density, const double *bx, const double *by,
                  const double *bz, const double *div_v, const double *curl_prev, const double *curl,
                  const double *curl_next, const double *l_turb_cm, double c_dens, double c_mag, double z_prev,
                  double z_curr, double z_next, int apply_temp_floor, int allow_curl_interp, int bfield_mode,
                  double mu_mol, double eta_B, double mach_limit, double l_turb_target_kpc, double *bg);

#ifdef __cplusplus
}
#endif
#endif
