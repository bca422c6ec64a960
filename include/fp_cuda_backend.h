/*
 * fp_cuda_backend.h -- the reference-compatible C ABI of the B200 library.
 *
 * These are the entry points, types and field orders of the CROMA CUDA
 * backend header include/fp_cuda_backend.h:1-165 (kosukenishiwaki/croma-fp),
 * with the nested input types of include/fp_shared_core.h and the momentum
 * grid of include/params.h.  CROMA's C host (include/tracer_fp_solve.inc,
 * src/tracer_fp.c, src/tracer_fp_entry_helpers.c) links
 * libcroma_b200_np<N>.so in place of the reference's fp_cuda_*.cu objects
 * without source changes; the bin count N must match the host's np == npe.
 *
 * Semantics follow the reference CPU backend where the reference's CPU and
 * CUDA paths differ (disable_adiabatic is honoured; the CC delta zeroing of
 * src/fp_shared_core.c:695 is applied).  Return codes: 0 success, -1
 * invalid argument or state, -2 numerical failure reported by a kernel, -3
 * CUDA error; nothing exits the process.  Model switches the reference
 * reads from CROMA's globals (dpp_mode_spec, ttd_tacc_model,
 * t_acc_direct_gyr, eta_dpp_cap; include/params.h) are read from the host
 * process when present and otherwise from croma_b200_set_model().
 */
#ifndef CROMA_B200_FP_CUDA_BACKEND_H
#define CROMA_B200_FP_CUDA_BACKEND_H

#ifndef np
#define np 128
#endif
#ifndef npe
#define npe 128
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* include/params.h:52-61 */
typedef struct {
    double p[np];
    double dp[np];
    double pp1;
    double pm1;
    double E[np];
    double N[np];
    double N_pre[np];
    double N_ave[np];
} CRspectrum;

/* include/fp_shared_core.h:366-407 */
typedef struct {
    int ncell;
    double z;
    double dt_gyr;
    double epmax;
    const double *n_gas;
    const double *kbt;
    const double *b_field;
    const double *divv_gyr;
    const unsigned char *disable_adiabatic;
    const double *l_turb_mpc;
    const double *dv_imc;
    const double *cs;
    const double *beta_pl;
    const double *tracer_mass_msun;
    const double *crp_state_cell_major;
    const double *cre_state_cell_major;
    const double *rad_ic_batch;      /* [npe * ncell] momentum-major */
    const double *rad_ic_m1;
    const double *rad_ic_p1;
    int device_interp_background;
    double interp_alpha;
    const double *n_gas_next;
    const double *kbt_next;
    const double *b_field_next;
    const double *divv_gyr_next;
    const double *l_turb_mpc_next;
    const double *dv_imc_next;
    const double *cs_next;
    const double *beta_pl_next;
    const double *rad_ic_batch_next;
    const double *rad_ic_m1_next;
    const double *rad_ic_p1_next;
} FpCoeffBatchInput;

/* include/fp_shared_core.h:466-489 */
typedef struct {
    int ncell;
    int nfreq;
    int nx_tab;
    int ntheta_pitch;
    int nlogb;
    double z;
    double xmin;
    double logb_min;
    double inv_dlogb;
    const double *fx_tab;
    const double *logfx_tab;
    const double *logx_tab;
    double ***logy;
    const double *pitch_kernel_table;  /* [nlogb * nfreq * npe] or NULL */
    const double *b_dyn;
    const double *logb;
    const double *cre_batch;           /* [ncell * npe] cell-major */
    const double *gamma2e;
    const double *theta;
    const double *dtheta;
    const double *pitch_weight;
    const double *nus;
} FpSynchEmissionBatchInput;

/* include/fp_shared_core.h:494-503 */
typedef struct {
    int ncell;
    int nbins;
    double z;
    double nu_min;                     /* log10(nu/Hz) */
    double nu_max;                     /* log10(nu/Hz) */
    const double *cre_batch;           /* [ncell * npe] cell-major */
    const double *fic_flat;            /* [nbins * npe] row-major */
} FpIcEmissionBatchInput;

/* include/fp_shared_core.h:502-514 */
typedef struct {
    int ncell;
    int nbins;
    double z;
    double egamma_min;
    double egamma_max;
    const double *n_gas;
    const double *crp_batch;           /* [ncell * np] cell-major */
    const double *beta_p;
    const double *fga_flat;            /* [nbins * np] row-major */
} FpGammaEmissionBatchInput;

/* include/fp_shared_core.h:516-528 */
typedef struct {
    int ncell;
    int nbins;
    double z;
    double enu_min;
    double enu_max;
    const double *n_gas;
    const double *crp_batch;
    const double *beta_p;
    const double *fnu_flat;
} FpNeutrinoEmissionBatchInput;

/* include/fp_shared_core.h:681-690 */
typedef struct {
    int nsys;
    int nrow;
    double dt;
    const double *a_batch;             /* [nsys * nrow] cell-major */
    const double *b_batch;
    const double *c_batch;
    const double *source_batch;
} FpChangCooperSolveBatchInput;

/* include/fp_cuda_backend.h:10 */
typedef struct FpCudaPipelineWorkspace FpCudaPipelineWorkspace;

/* include/fp_cuda_backend.h:12-20 */
typedef struct {
    int emit_final_only;
    int emit_all_steps;
    int emit_stride;
    int physical_min;
    int physical_max;
    const int *selected_steps;
    int nselected_steps;
} FpCudaOutputSchedule;

/* include/fp_cuda_backend.h:22-25 */
typedef enum {
    FP_CUDA_TRANSPORT_LEGACY = 0,
    FP_CUDA_TRANSPORT_FUSED_SUBSTEPS = 1
} FpCudaTransportMode;

/* include/fp_cuda_backend.h:27-67 */
typedef struct {
    int ncell;
    int nstep;
    int fp_cadence_steps;
    int diff_cadence_steps;
    int adv_cadence_steps;
    int use_windowed_reacc;
    int on_start_step;
    int on_end_step;
    int nfreq;
    int nx_tab;
    double dt;
    double epmax;
    double xmin;
    double psi_value;
    double mach_limit_value;
    FpCudaTransportMode transport_mode;
    const CRspectrum *crp_grid;
    const CRspectrum *cre_grid;
    const FpCoeffBatchInput *coeff_in;
    const FpSynchEmissionBatchInput *synch_in;
    const FpGammaEmissionBatchInput *gamma_in;
    const FpNeutrinoEmissionBatchInput *neutrino_in;
    const double *qpi_batch;           /* [ncell * np ] cell-major */
    const double *qepri_batch;         /* [ncell * npe] cell-major */
    const double *beta_p;              /* [np] */
    const double *crp_init;            /* [ncell * np ] cell-major */
    const double *cre_init;            /* [ncell * npe] cell-major */
    double *crp_state_out;
    double *cre_state_out;
    double *eps_syn_out;
    double *eps_gamma_out;
    double *eps_nu_out;
    const int *rank_state_indices;     /* [ncell] rank-local tracer indices */
    int gather_rank_state;
    int scatter_rank_state;
    FpCudaPipelineWorkspace *workspace;
} FpCudaPipelineInput;

/* include/fp_cuda_backend.h:69-90 */
typedef struct {
    double setup_ms;
    double h2d_ms;
    double device_interp_ms;
    double coeff_ms;
    double secondary_ms;
    double solve_ms;
    double diff_ms;
    double adv_ms;
    double synch_ms;
    double gamma_ms;
    double neutrino_ms;
    double d2h_ms;
    double other_ms;
    double total_ms;
    int emitted_synch;
    int emitted_gamma;
    int emitted_neutrino;
    int last_synch_step;
    int used_pcr_proton;
    int used_pcr_electron;
} FpCudaPipelineTimes;

/* ---- entry points: include/fp_cuda_backend.h:92-159 ---- */
int cuda_pipeline_is_available(void);                                        /* :92  */
int cuda_bind_local_rank(int local_rank, int *device_out);                   /* :93  */
int cuda_get_binding_state(int *device_count_out, int *current_device_out);  /* :94  */
int cuda_get_current_device_id(char *device_id_out, int device_id_out_len);  /* :95  */

int prepare_synch_emission_cuda_batch(const FpSynchEmissionBatchInput *in,   /* :97-100 */
                                      const CRspectrum *cre_grid,
                                      double *eps_syn_out,
                                      double *elapsed_ms);
/* Both branches of prepare_synch_emission_cell_major
 * (src/fp_shared_core.c:2070-2129): with in->pitch_kernel_table (nlogb > 1,
 * inv_dlogb > 0) the log-K interpolation of the table; without it the
 * pitch-angle integral of SYN_emissivity_from_arrays (src/Synchrotron.c:62-103)
 * from fx_tab / logfx_tab / logx_tab / logy / pitch_weight. */

/* The device form of the host routine prepare_synch_pitch_kernel_table
 * (src/fp_shared_core.c:2008-2052), which tracer_fp_refresh_synch_kernel_table
 * (src/tracer_fp_synch.c:175-240) calls on every log B range refresh:
 * kernel_table[(ib * nfreq + nf) * npe + je] = sum_k F(logy[nf][je][k] - logb_ib)
 * pitch_weight[k], logb_ib = logb_min + ib / inv_dlogb, written to the host
 * array kernel_table [nlogb * nfreq * npe]. */
int prepare_synch_pitch_kernel_table_cuda(const FpSynchEmissionBatchInput *in,
                                          double *kernel_table,
                                          double *elapsed_ms);
/* The device form of the CPU routine prepare_ic_emission_batch
 * (src/fp_shared_core.c:2131-2164), which the reference's CUDA backend does not
 * provide: eps_ic[cell][band] = sum_je fic[band][je] N[cell][je] dp[je]. */
int prepare_ic_emission_cuda_batch(const FpIcEmissionBatchInput *in,
                                   const CRspectrum *cre_grid,
                                   double *eps_ic_out,
                                   double *elapsed_ms);
/* Device forms of the host routines that build the emission kernel tables
 * (no CUDA counterpart in the reference; its CPU code builds them once per
 * run, the IC table once per emitted snapshot).  Host grid in, host table
 * out, [nbins][np] (gamma, neutrino: proton grid) or [nbins][npe] (IC:
 * electron grid), band k at 10^(lo + k d), d = (hi - lo) / nbins, accumulated
 * as the reference does.
 *   prepare_gamma_kernel_flat     src/fp_shared_core.c:1724-1749 (gammaKernel, src/HADRONIC.c:139-177)
 *   prepare_neutrino_kernel_flat  src/fp_shared_core.c:1751-1778 (eKernel + numu1Kernel, src/HADRONIC.c:181-289)
 *   prepare_ic_kernel_flat        src/fp_shared_core.c:1780-1807 (IC_emissivity_kernel, src/FP_Coef.c:553-584) */
int prepare_gamma_kernel_flat_cuda(const CRspectrum *crp, int nbins, double egamma_min, double egamma_max,
                                   double *fga_flat);
int prepare_neutrino_kernel_flat_cuda(const CRspectrum *crp, int nbins, double enu_min, double enu_max,
                                      double *fnu_flat);
int prepare_ic_kernel_flat_cuda(const CRspectrum *cre, int nbins, double nu_min, double nu_max, double z,
                                double *fic_flat);
/* The log10 F(x) column of SYN_logFx_table (src/Synchrotron.c:31-41) on the
 * device: F(x) = x int_x^inf K_5/3(s) ds for x <= 300 from the integral
 * definition (the reference calls GNU GSL's gsl_sf_synchrotron_1 there; GSL
 * is not part of this library), sqrt(pi/2) exp(-x) sqrt(x) above, as the
 * reference does. */
int synch_logfx_table_cuda(int nx, const double *logx, double *logfx_out);

int prepare_gamma_emission_cuda_batch(const FpGammaEmissionBatchInput *in,   /* :102-105 */
                                      const CRspectrum *crp_grid,
                                      double *eps_gamma_out,
                                      double *elapsed_ms);
int prepare_neutrino_emission_cuda_batch(const FpNeutrinoEmissionBatchInput *in, /* :107-110 */
                                         const CRspectrum *crp_grid,
                                         double *eps_nu_out,
                                         double *elapsed_ms);

int solve_cc_cuda_batch(const FpChangCooperSolveBatchInput *in,             /* :112-116 */
                        const double *state_init,
                        double *state_out,
                        double *elapsed_ms,
                        int *used_pcr_out);

/* No counterpart in the reference.  The same implicit Chang-Cooper step as
 * solve_cc_cuda_batch for callers that must not allocate device memory (a
 * host whose device memory already belongs to its own pool allocator, or a
 * time step that cannot afford cudaMalloc/cudaFree synchronising the device):
 * every pointer is a device pointer owned by the caller, layout
 * [nsys][nrow] as in FpChangCooperSolveBatchInput, stream is a cudaStream_t
 * (0 for the default stream).  The only scratch is a fixed array inside the
 * library, so nsys * nrow may not exceed 524288 (larger batches return -1);
 * every GPU that loads the library keeps that 4 MiB array until exit.  All
 * calls on a device share it: calls that overlap on the GPU race and must be
 * serialised.  The first call on a device looks the array up and caches its
 * address; the stream must belong to the current device (-1 otherwise), and
 * after a cudaDeviceReset the library is not to be used on that device.  The
 * call waits for its stream and returns -2 on a singular pivot; because of
 * that wait it refuses (-1, nothing launched) a stream that is being
 * captured. */
int solve_cc_cuda_batch_noalloc(int nsys, int nrow, double dt,
                                const double *a, const double *b, const double *c,
                                const double *source, const double *state_in,
                                double *state_out, void *stream);

int fp_cuda_tridiag_uses_pcr(int nrow);                                      /* :118 */
const char *fp_cuda_tridiag_solver_name(int nrow);                           /* :119 */

FpCudaPipelineWorkspace *cuda_pipeline_workspace_create(void);               /* :121 */
void cuda_pipeline_workspace_destroy(FpCudaPipelineWorkspace *workspace);    /* :122 */

int cuda_rank_state_upload(FpCudaPipelineWorkspace *workspace,               /* :124-130 */
                           int ncell,
                           const double *qpi,
                           const double *qepri,
                           const double *crp,
                           const double *cre,
                           double *elapsed_ms);
int cuda_rank_state_download(FpCudaPipelineWorkspace *workspace,             /* :132-136 */
                             int ncell,
                             double *crp,
                             double *cre,
                             double *elapsed_ms);

int run_tracer_pipeline(const FpCudaPipelineInput *in,                       /* :138-145 */
                        const FpCudaOutputSchedule *schedule,
                        double *crp_state_out,
                        double *cre_state_out,
                        double *eps_syn_out,
                        double *eps_gamma_out,
                        double *eps_nu_out,
                        FpCudaPipelineTimes *times);
int run_tracer_pipeline_group(const FpCudaPipelineInput *inputs,             /* :147-150 */
                              int ninput,
                              const FpCudaOutputSchedule *schedule,
                              FpCudaPipelineTimes *times);
/* Declared but never defined by the reference (:152-159); here it runs the
 * same pipeline as run_tracer_pipeline. */
int run_pipeline_cuda(const FpCudaPipelineInput *in,
                      const FpCudaOutputSchedule *schedule,
                      double *crp_state_out,
                      double *cre_state_out,
                      double *eps_syn_out,
                      double *eps_gamma_out,
                      double *eps_nu_out,
                      FpCudaPipelineTimes *times);

/* Model switches for standalone use (no counterpart in the reference,
 * whose backend reads them from CROMA's globals): Dpp model as
 * FP_MOMENTUMDIFF_MODEL_* (1 ASA, 2 TTD, 3 off, 4 direct_tacc),
 * ttd_tacc_model (0 spectral, 1 brunetti16), direct t_acc [Gyr] and the
 * eta cap.  When CROMA's own globals are linked in they take precedence. */
int croma_b200_set_model(int dpp_model, int ttd_tacc_model, double t_acc_direct_gyr,
                         double eta_dpp_cap);

#ifdef __cplusplus
}
#endif
#endif
