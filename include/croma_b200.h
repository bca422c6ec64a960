/*
 * croma_b200.h -- native C ABI of the B200 tracer Fokker-Planck library
 * (libcroma_b200_np<N>.so, N = bins per species: 128, 256 or 512).
 *
 * This is the batched, device-resident form of the per-snapshot sequence
 * that the reference's snapshot driver runs for the tracer FP update
 * (include/tracer_fp_solve.inc in kosukenishiwaki/croma-fp):
 *
 *   IC-cooling rows   tracer_fp_prepare_ic_cooling_snapshot (src/tracer_fp_synch.c:242-294)
 *   nsub / n_on       tracer_fp_prepare_nsub_loss_endpoints + tracer_fp_compute_nsubsteps_from_endpoints
 *                     (src/tracer_fp_nsub.c:94-282)
 *   buckets           tracer_bucket_build_snapshot (src/tracer_fp_bucket.c:208-262)
 *   evolve            tracer_fp_batch_execute_parallel / run_tracer_pipeline
 *                     (src/tracer_fp_batch.c:651-1126, src/fp_cuda_tracer_backend.cu:1530-1567)
 *
 * The reference-compatible entry points (run_tracer_pipeline and friends)
 * are declared in fp_cuda_backend.h and implemented on the same kernels.
 *
 * All functions return 0 on success and a negative code on failure
 * (-1 invalid argument or state, -2 numerical failure reported by a kernel,
 * -3 CUDA error, -4 allocation failure); they never exit the process.
 * croma_b200_last_error() describes the last failure of the calling thread.
 * Pointers are plain host or device addresses as stated per argument.
 */
#ifndef CROMA_B200_H
#define CROMA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CromaB200Context CromaB200Context;

/* Dpp_mode values (FP_MOMENTUMDIFF_MODEL_*, include/fp_shared_core.h:227-233). */
enum { CROMA_DPP_ASA = 1, CROMA_DPP_TTD = 2, CROMA_DPP_OFF = 3, CROMA_DPP_DIRECT_TACC = 4 };

/* Which evolve kernel family runs. */
enum {
    CROMA_PATH_PLAIN = 0,   /* FP64, reference data contract: CC rows materialised per
                               segment, every sub-step reads them, the source and N
                               from memory, re-pivots and writes N (per-step) */
    CROMA_PATH_FUSED = 1,   /* FP64, on-chip: rows built, factored and swept per tracer
                               inside one kernel, warp-cooperative substitution */
    CROMA_PATH_FUSED_FP32R = 2  /* the on-chip path with each sub-step solved in FP32 and
                               refined once with an FP64 residual (FP64 factors, CC
                               weights, spectra and particle budget) */
};

/* Species bits: bit 0 protons, bit 1 electrons.  A species outside the mask
 * must have zero spectra and zero source; it is then left untouched, which
 * is exactly what the implicit solve returns for it.  The reference evolves
 * both species whatever its seed (seed_cr_species): an electron-only seed
 * maps to mask 2, a proton or mixed seed to mask 3 (protons feed secondary
 * electrons).  Mask 1 skips the electrons, secondaries included. */
enum { CROMA_SPECIES_PROTON = 1, CROMA_SPECIES_ELECTRON = 2 };

typedef struct {
    int nb;                          /* bins per species; must equal the library's N */
    int species_mask;
    double pmin, pmax;               /* log10 proton grid bounds (params.c:55) */
    double pemin, pemax;             /* log10 electron grid bounds (params.c:56) */
    int dpp_model;                   /* CROMA_DPP_* */
    int ttd_tacc_model;              /* 0 spectral, 1 brunetti16 (params.c:74-75) */
    double t_acc_direct_gyr;
    double mach_limit;               /* params.c:77 */
    double psi;                      /* params.c:76 */
    double eta_dpp_cap;              /* params.c:78; <= 0 disables */
    double nsub_safety;              /* tracer_nsub_safety, params.c:83 */
    int nsub_max;                    /* tracer_nsub_max; 0 = no cap */
    int coeff_interp_min_steps;      /* params.c:85 */
    int coeff_interp_max_segments;   /* params.c:86 */
    int reacc_window_mode;           /* 0 always on, 1 centred */
    double f_eddy;
    double t_off_gyr;
    double t_acc_off_gyr;
    int path;                        /* CROMA_PATH_* */
} CromaB200Config;

typedef struct {
    const double *bg_curr;   /* [8][ntracer] field-major: n_gas, kbt, b_field, divv_gyr,
                                l_turb_mpc, dv_imc, cs, beta_pl (the TracerFpBackgroundSlot
                                fields of include/tracer_fp_types.h) */
    const double *bg_next;   /* same for the next snapshot (ignored unless allow_interp) */
    int bg_on_device;        /* 1: device pointers, 0: host pointers */
    double z_curr, z_next;
    int allow_interp;        /* background interpolation across the snapshot */
    double dt_snap;          /* Gyr */
    double elapsed_gyr;      /* time at the start of the snapshot */
} CromaB200Snapshot;

const char *croma_b200_last_error(void);
int croma_b200_nb(void);                       /* bins per species compiled into this library */

int croma_b200_create(const CromaB200Config *cfg, int device, CromaB200Context **out);
void croma_b200_destroy(CromaB200Context *ctx);

/* Device workspace and state for up to ntracer tracers. */
int croma_b200_reserve(CromaB200Context *ctx, int ntracer);

/* Cap (device bytes) on the evolve workspace (either path); tracers beyond
 * what it holds run in chunks.  Takes effect at the next reserve; 0 restores
 * the default (CROMA_B200_WORKSPACE_GB, else 24 GB). */
int croma_b200_set_workspace_limit(CromaB200Context *ctx, double bytes);

/* Host <-> device spectra, cell-major host arrays [ntracer][nb] (the
 * reference's layout).  NULL skips an array; sources default to zero. */
int croma_b200_set_state(CromaB200Context *ctx, int ntracer, const double *crp,
                         const double *cre, const double *qpi, const double *qepri,
                         const double *mass_msun, const unsigned char *disable_adiabatic);
int croma_b200_get_state(CromaB200Context *ctx, double *crp, double *cre);
/* Every tracer starts from the same seed spectra (host rows [nb]) and mass, as
 * the reference's seed initialisation gives them; sources and flags zero. */
int croma_b200_set_state_broadcast(CromaB200Context *ctx, int ntracer, const double *crp_row,
                                   const double *cre_row, double mass_msun);
/* The resident sources (cell-major host arrays [ntracer][nb]) and the
 * disable-adiabatic flags [ntracer]; NULL skips an array. */
int croma_b200_get_sources(CromaB200Context *ctx, double *qpi, double *qepri, unsigned char *dis);

/* Scheduling priority of the context's stream (CUDA stream priorities: lower
 * numbers run first; clamped to cudaDeviceGetStreamPriorityRange).  Waits
 * for the context's queued work and replaces its stream.  The request server
 * gives small requests the higher priorities so that their blocks are
 * scheduled ahead of the remaining blocks of large requests' kernels. */
int croma_b200_set_priority(CromaB200Context *ctx, int priority);

/* One snapshot on the context's stream; asynchronous unless sync != 0. */
int croma_b200_snapshot(CromaB200Context *ctx, const CromaB200Snapshot *snap, int sync);

/* One snapshot from host spectra to host spectra: the same result and
 * resident state as set_state(crp, cre, NULL, NULL, mass, NULL), snapshot,
 * get_state(crp, cre), with the copies overlapped with the evolve.  The
 * tracers run in chunks: the upload of later chunks and the download of
 * earlier ones proceed on two copy streams while a chunk is evolved.
 * crp / cre ([ntracer][nb], cell-major) are read and overwritten with the
 * evolved spectra; a species the mask does not evolve is not copied back.
 * Page-locked host memory is needed for the copies to overlap.
 * chunks <= 0: an eighth of the tracers at each end and the middle in
 * workspace-sized pieces; otherwise that many near-equal chunks.
 * Synchronous: returns after the last download. */
int croma_b200_snapshot_host(CromaB200Context *ctx, const CromaB200Snapshot *snap, int ntracer,
                             double *crp, double *cre, const double *mass_msun, int chunks);

/* Schedule of the last snapshot (host arrays of ntracer ints); NULL skips. */
int croma_b200_get_schedule(CromaB200Context *ctx, int *nsub, int *n_on, int *target_nsub,
                            int *bucket_ids, int *bucket_indices, int *nbuckets);

/* IC-cooling row for one redshift (host output: row[nb], then m1, p1). */
int croma_b200_ic_row(CromaB200Context *ctx, double z, double *row_m1_p1);

/* Grid and one-time tables (host outputs): p, dp, E [nb] then pm1, pp1. */
int croma_b200_get_grid(CromaB200Context *ctx, int species, double *out);
int croma_b200_get_secondary_kernel(CromaB200Context *ctx, double *fqe_flat, int *np_min_qe);

/* The context's CUDA stream (cudaStream_t) and a blocking wait on it. */
void *croma_b200_stream(CromaB200Context *ctx);
int croma_b200_sync(CromaB200Context *ctx);

/* Device pointers of the resident spectra, momentum-major [nb][ntracer]. */
int croma_b200_state_device(CromaB200Context *ctx, double **crp, double **cre);

/* Kernel launches issued by the last croma_b200_snapshot call. */
int croma_b200_last_launch_count(CromaB200Context *ctx);

/* Optional per-kernel timing with CUDA events on the context stream.
 * kind: 0 evolve (sub-step) kernels, 1 coefficient kernels, 2 secondary
 * source kernels.  kernel_stats waits for the stream and returns the
 * accumulated device time and launch count since the last reset. */
int croma_b200_set_kernel_timing(CromaB200Context *ctx, int enable);
int croma_b200_kernel_stats(CromaB200Context *ctx, int kind, double *total_ms, long long *launches);
int croma_b200_reset_kernel_stats(CromaB200Context *ctx);

/* ---- DSA (diffusive shock acceleration) injection ----
 * The per-snapshot shock injection of tracer_fp_apply_dsa_tracer_injection_snapshot
 * (src/tracer_fp_dsa.c:184-565), run on the resident spectra.  Parameters
 * mirror the reference's globals (src/params.c:96-113, mu_mol :127) and the
 * DSA grid bounds passed to dsa_init_grid (src/tracer_fp.c:841).  Model ids
 * follow DSAModelID: 0 KR07, 1 KR07r, 2 KR13, 3 KR13r, 4 CS14, 5 CS14r,
 * 6 Ryu19, 7 Ryu19r. */
typedef struct {
    int eta_model_initial, eta_model_reacc;
    double chi_p, chi_e, k_ep, pmax_p_mc, pmax_e_mc;
    double min_mach, gamma_gas, xcr_pmin_pmc, reacc_eta_cap, mu_mol;
    double pmin_dsa_p_log10, pmin_dsa_e_log10;
    int inject_species;              /* 0 both, 1 electrons, 2 protons */
} CromaB200DsaParams;

/* Shock fields of every resident tracer ([ntracer] each; NULL = absent), the
 * TracerFpRawBackgroundSlot fields of include/tracer_fp_types.h:292-313. */
typedef struct {
    const double *mach, *prestemp, *presden, *pre_density_cgs, *upstream_speed_cgs, *shock_side_code;
    const double *dsa_trigger, *dsa_mach, *dsa_pre_density, *dsa_flux_cgs;
    int has_dsa;                     /* 1: merged-DSA fields, 0: raw shock fields */
    int on_device;                   /* 1: device pointers, 0: host pointers */
} CromaB200Shocks;

enum { CROMA_DSA_OFF = 0, CROMA_DSA_TRACER_STATE = 1, CROMA_DSA_TRACER_SOURCE = 2 };
enum { CROMA_DSA_REACC_OFF = 0, CROMA_DSA_REACC_POSITIVE_DELTA = 1, CROMA_DSA_REACC_DRURY83 = 2 };

int croma_b200_set_dsa(CromaB200Context *ctx, const CromaB200DsaParams *params);

/* One snapshot's injection, before croma_b200_snapshot.  tracer_state adds
 * source x V_down to the spectra; tracer_source replaces the sources with
 * source x V_down / dt_gyr (they start from zero, as in the reference's
 * snapshot driver).  The disable-adiabatic flags are cleared and set for the
 * tracers drury83 reaccelerates.  A species that receives particles joins the
 * context's species mask (the reference always evolves both species).
 * Synchronous; *ninjected (may be NULL) receives the number of tracers
 * injected. */
int croma_b200_dsa_inject(CromaB200Context *ctx, const CromaB200Shocks *shocks, double density_unit,
                          double dt_gyr, int mode, int reacc_mode, int *ninjected);

/* ---- Emissivities of the resident spectra ----
 * The per-snapshot emission integrals of the reference ABI
 * (prepare_ic_emission_cuda_batch, prepare_gamma/neutrino_emission_cuda_batch,
 * prepare_synch_emission_cuda_batch with a pitch-kernel table; include/
 * fp_cuda_backend.h:97-110 of the reference) computed on the spectra the
 * context already holds on the device, one row per tracer in the context's
 * tracer order, with the same kernels and results bit for bit.  Only the
 * kernel tables and per-tracer inputs (host arrays) go to the device and the
 * emissivities (host arrays [ntracer][ncols]) come back: the spectra
 * themselves do not cross PCIe.  Synchronous; *elapsed_ms (may be NULL)
 * receives the device time of the call, copies included.  Errors: -1 invalid
 * (no resident state, a species the context does not evolve, missing
 * inputs), -3 CUDA. */

/* eps[t][band] = sum_je fic[band][je] N_e[t][je] dp_e[je]; fic [nbands][nb]. */
int croma_b200_emission_ic(CromaB200Context *ctx, int nbands, const double *fic, double *eps_out,
                           double *elapsed_ms);

/* Hadronic gamma or neutrino emission of the proton spectra:
 * eps[t][bin] = E_bin n_gas[t] 1/2 sum_i (f_{i-1} + f_i) dp_i,
 * f_i = beta_p[i] N_p[t][i] kernel[bin][i], E_bin log-spaced over
 * [e_min, e_max] as the reference accumulates it; kernel is the gamma or the
 * neutrino table [nbins][nb]; n_gas [ntracer], beta_p [nb]. */
int croma_b200_emission_hadronic(CromaB200Context *ctx, int nbins, double e_min, double e_max,
                                 const double *n_gas, const double *beta_p, const double *kernel,
                                 double *eps_out, double *elapsed_ms);

/* Synchrotron emission of the electron spectra through the pitch-kernel
 * table [nlogb][nfreq][nb] (log-K interpolation in log B, nlogb > 1,
 * inv_dlogb > 0); b_dyn and logb [ntracer]. */
int croma_b200_emission_synch(CromaB200Context *ctx, int nfreq, int nlogb, double logb_min, double inv_dlogb,
                              const double *table, const double *b_dyn, const double *logb, double *eps_out,
                              double *elapsed_ms);

/* ---- Emission of the resident spectra into device memory ----
 * The per-snapshot emission of the reference's snapshot driver
 * (include/tracer_fp_solve.inc:117-426: synchrotron, inverse Compton,
 * hadronic gamma rays and neutrinos, from the spectra the snapshot starts
 * from) with every kernel table built on the device:
 *   F(x) = x int_x^inf K_5/3 from its integral definition (the reference
 *   calls GNU GSL's gsl_sf_synchrotron_1 in SYN_logFx_table,
 *   src/Synchrotron.c:31-41), the 2750-point log-x grid, pitch angles,
 *   frequencies, logy and the log-B pitch-kernel table of
 *   tracer_fp_synch_data_init_tables / tracer_fp_refresh_synch_kernel_table
 *   (src/tracer_fp_synch.c:87-121, 175-240, fixed log-B range);
 *   the gamma / neutrino tables of prepare_gamma/neutrino_kernel_flat
 *   (src/fp_shared_core.c:1724-1778), once;
 *   the IC table of prepare_ic_kernel_flat (:1780-1807), rebuilt when z changes.
 * Band grids follow the reference: band k at 10^(lo + (k+1) d - d),
 * d = (hi - lo) / nbins, lo / hi in log10 Hz (synchrotron, IC) or log10 GeV
 * (gamma, neutrino).  A count of 0 disables that kind. */
typedef struct {
    int nfreq;                         /* synchrotron frequencies */
    double nu_min_s, nu_max_s;         /* log10 Hz (params.c:116 defaults 5.5, 10.5) */
    int ntheta_pitch;                  /* pitch angles (N_theta_pitch, params.h:12: 512) */
    int nlogb;                         /* log-B planes (TRACER_FP_SYNCH_LOGB_BINS: 512) */
    double logb_min, logb_max;         /* log10(B / 1 uG) range (params.c:117: -6, 2) */
    int nbins_ic;
    double nu_min_ic, nu_max_ic;       /* log10 Hz (params.c:120: 13, 28) */
    int nbins_gamma;
    double egamma_min, egamma_max;     /* log10 GeV (params.c:121: -2, 6) */
    int nbins_nu;
    double enu_min, enu_max;           /* log10 GeV (params.c:122: -2, 8) */
} CromaB200EmissionSetup;

/* Builds the tables on the device (synchronous).  Errors: -1 invalid setup
 * (a kind whose species the context does not evolve), -3 CUDA. */
int croma_b200_emission_setup(CromaB200Context *ctx, const CromaB200EmissionSetup *setup);

/* Emissivities of the resident spectra at redshift z: eps_* [ntracer][bins of
 * the kind], NULL skips a kind.  bg is the snapshot's background block
 * ([8][ntracer] field-major as in CromaB200Snapshot): n_gas (field 0) scales
 * the hadronic kinds, B (field 2) is the synchrotron b_dyn.  on_device = 1:
 * bg and the outputs are device pointers and the call is asynchronous on the
 * context stream (the outputs are ready when croma_b200_sync returns);
 * on_device = 0: host pointers, synchronous.  Results agree with the
 * reference's prepare_*_emission_cell_major on the same tables to rounding
 * (the sums run in another order). */
int croma_b200_emission_run(CromaB200Context *ctx, const double *bg, double z, double *eps_syn,
                            double *eps_ic, double *eps_gamma, double *eps_nu, int on_device);

/* A table of the emission setup, copied to host memory: which =
 * CROMA_EMIS_TABLE_SYNCH the pitch-kernel table [nlogb][nfreq][nb],
 * CROMA_EMIS_TABLE_IC the IC table [nbins_ic][nb] of the last run's z. */
enum { CROMA_EMIS_TABLE_SYNCH = 0, CROMA_EMIS_TABLE_IC = 1 };
int croma_b200_emission_table(CromaB200Context *ctx, int which, double *out);

/* One snapshot step of the resident pipeline through host memory: the
 * per-snapshot sequence of the reference's driver (include/tracer_fp_solve.inc:
 * DSA injection :76-101, emission :117-426, evolve :677-1526) with the
 * snapshot's inputs (backgrounds, shock fields) read from host memory and its
 * outputs (emissivities, evolved spectra) written to host memory, while the
 * spectra stay resident.  The emissivities come back on a copy stream while
 * the evolve runs, the evolved spectra workspace chunk by workspace chunk as
 * each finishes; page-locked host buffers let the copies overlap.
 * snap: host backgrounds (bg_on_device = 0).  Synchronous. */
typedef struct {
    const CromaB200Shocks *shocks;     /* host shock fields; NULL or dsa_mode OFF: no injection */
    int dsa_mode, dsa_reacc;           /* CROMA_DSA_*, CROMA_DSA_REACC_* */
    double density_unit;
    double *eps_syn, *eps_ic, *eps_gamma, *eps_nu;   /* host [ntracer][bins] or NULL */
    double *crp_out, *cre_out;                        /* host [ntracer][nb] or NULL */
} CromaB200StepHost;
int croma_b200_step_host(CromaB200Context *ctx, const CromaB200Snapshot *snap, const CromaB200StepHost *io);

/* The steps-kernel autotuner (the on-chip FP64 path).  The arithmetic is
 * fixed by rule, so that no result depends on a timing: the short-chain warp
 * scan (radix-4 warp scans, the back substitution's local pass overlapping
 * the forward scan) at 512 bins and more, the warp scan below, warp PCR (one
 * warp per tracer, parallel cyclic reduction in shared memory) when
 * CROMA_CUDA_TRIDIAG=pcr (src/fp_cuda_solver.cu:41-72 of the reference).
 * Within that family the variants compute bit-identical results and differ
 * in where the per-segment constants live -- registers, partly shared memory
 * (fewer registers, more warps per SM), or with each row's right-hand-side
 * scaling in shared memory too -- and in tracers (warps) per block, 1 or 2.
 * On the first workspace chunk a context evolves, per species, each of them
 * runs the chunk's first tracers (up to 16,384, several full waves of every
 * variant) for 16 sub-steps on a copy of their spectra, timed with CUDA
 * events, and the fastest is kept for the context; a calibration on the full
 * 16,384 tracers is reused by the process's later contexts (same species,
 * source and CROMA_CUDA_TRIDIAG).  Reported here: tuned (0 before the first
 * snapshot), solver (0 scan, 1 FP32-refined scan, 2 PCR, 3 scan with
 * shared-memory constants, 4 scan with the right-hand-side scaling in shared
 * memory, 5 short-chain scan), tracers per block, and the calibration time of
 * each variant in milliseconds, variant_ms[CROMA_B200_STEPS_VARIANTS] in the
 * order scan x1, scan x2, shared scan x1, shared scan x2, PCR, rhs-shared
 * scan x1, rhs-shared scan x2, short-chain scan x1, short-chain scan x2
 * (-1 = not run).  CROMA_B200_STEPS_VARIANT=0..8 fixes the variant in that
 * order without calibrating (reproducible profiles). */
#define CROMA_B200_STEPS_VARIANTS 9
int croma_b200_get_tuning(CromaB200Context *ctx, int species, int *tuned, int *solver, int *warps_per_block,
                          double *variant_ms);

/* Page-locked host memory of exactly `bytes` (cudaHostAlloc, portable), for
 * the host-buffer calls above, whose copies overlap the kernels only from
 * page-locked memory; released by croma_b200_host_free (which waits for the
 * device). */
int croma_b200_host_alloc(size_t bytes, void **out);
int croma_b200_host_free(void *p);

/* ---- tracer snapshots from HDF5 and their backgrounds ---------------- */

/* Reader of the HDF5 tracer snapshots CROMA takes as input (the reference
 * reads them with libhdf5: tracer_load_hdf5_raw_snapshot_slice,
 * src/tracer_fp_background.c:1003-1204).  It reads the format subset those
 * files use -- superblock 0/1, symbol-table groups, version-1 object
 * headers, compact or contiguous datasets of fixed-point or IEEE
 * floating-point elements -- and refuses the rest with an error naming it.
 * dataset may be a '/'-separated path.  h5_shape: rank, up to max_rank
 * dimensions, datatype class (0 fixed-point, 1 floating-point) and element
 * size.  h5_read_f64 / _i64: elements [offset, offset + count) of the
 * dataset in storage order, converted to double / int64 (_i64 only for
 * fixed-point datasets). */
int croma_b200_h5_shape(const char *path, const char *dataset, int *rank, long long *dims, int max_rank,
                        int *type_class, int *type_size);
int croma_b200_h5_read_f64(const char *path, const char *dataset, long long offset, long long count, double *out);
int croma_b200_h5_read_i64(const char *path, const char *dataset, long long offset, long long count,
                           long long *out);

/* The raw fields of one tracer snapshot, as the snapshot files hold them:
 * temperature [K], density [code units], B_x/y/z [code units], div_v and
 * curl_v [s^-1] (curl_v also of the previous and next snapshots when
 * allow_curl_interp), dx_phys [cm] (NULL or <= 0: the target scale), and the
 * snapshot's unit factors c_dens = dUnit and c_mag = sqrt(4 pi dUnit) vUnit
 * (src/tracer_fp_background.c:955-957, 1189-1197). */
typedef struct {
    const double *temp_K, *density, *bx, *by, *bz, *div_v;
    const double *curl_v_prev, *curl_v, *curl_v_next;
    const double *l_turb_cm;
    double c_dens, c_mag;
    double z_prev, z_curr, z_next;
    int apply_temp_floor;    /* T < 1e4 K -> 1e4 K */
    int allow_curl_interp;   /* curl_v == 0 -> interpolated in z from prev / next */
} CromaB200RawSnapshot;

/* The run parameters the background reads (src/params.c): bfield_mode
 * 0 max(dynamo, simulation), 1 simulation, 2 dynamo; mu_mol 0.59; eta_B
 * 0.05; mach_limit 0.5; L_turb_target_kpc 150 are the reference's defaults. */
typedef struct {
    int bfield_mode;
    double mu_mol, eta_B, mach_limit, l_turb_target_kpc;
} CromaB200BackgroundParams;

/* The background block [8][ntracer] (n_gas, kT GeV, B_eff, div v Gyr^-1,
 * L_turb Mpc, dv_imc, c_s, beta_pl) that croma_b200_snapshot reads, from one
 * snapshot's raw fields: prepare_background_cell (src/fp_shared_core.c:866-932)
 * per tracer, as tracer_prepare_background_from_raw (src/tracer_fp_background.c:
 * 1206-1263) applies it, one device thread per tracer.  on_device: raw arrays
 * and bg are device pointers (else host).  ctx (may be NULL) supplies the
 * stream.  Returns 0, -1 on invalid arguments or a CUDA error, -2 when a
 * tracer has density <= 0 (the reference aborts; its fields are set to 0). */
int croma_b200_background_prepare(CromaB200Context *ctx, int ntracer, const CromaB200RawSnapshot *raw,
                                  const CromaB200BackgroundParams *prm, int on_device, double *bg);

/* FP64 FMA throughput of the current device, measured by a kernel of
 * independent fused multiply-add chains on every SM (TFLOP/s, FMA = 2 flops);
 * the denominator of the fused evolve's roofline. */
int croma_b200_fp64_peak(double *tflops);

/* The device reciprocal of the factor and per-step kernels (an inline
 * rcp.approx.ftz.f64 refined by two Newton-Raphson steps) applied to n host
 * doubles x on the current device, for checking its error bound. */
int croma_b200_rcp_check(long long n, const double *x, double *out);
/* The same for the factor kernels' table-driven exponential. */
int croma_b200_exp_check(long long n, const double *x, double *out);

#ifdef __cplusplus
}
#endif
#endif
