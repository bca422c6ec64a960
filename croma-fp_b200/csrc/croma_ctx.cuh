// croma_ctx.cuh -- the library context: device tables, resident state,
// workspaces and the per-snapshot schedule.  Internal header.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/croma_b200.h"
#include "croma_phys.cuh"

#ifndef CROMA_NB
#error "CROMA_NB (bins per species) must be defined at compile time"
#endif

namespace croma {

struct EmissionState;   // emission.cu

constexpr int NB = CROMA_NB;
static_assert(NB == 128 || NB == 256 || NB == 512, "supported bin counts: 128, 256, 512");

constexpr int kNbg = 8;   // background fields per tracer
// One IC slot: the row (nb), its ghost edges (2), then scratch for the
// outer CMB abscissae of b_IC (up to 2049 points).
constexpr int kIcSlotDoubles = NB + 2 + 2049;

// Per-tracer schedule written by the sub-step estimator.
struct Schedule {
    int *nsub, *non, *target, *nseg;
    unsigned char *capped;
    int *bucket_ids, *bucket_indices;
    int *nbuckets;            // device scalar
};

// Everything a snapshot kernel needs, passed by value.
struct SnapArgs {
    int ntracer;
    const double *bg_curr, *bg_next;   // [8][ntracer]
    const double *ic_curr, *ic_next;   // [nb+2] each
    int allow_interp;
    double dt_snap, elapsed;
    double *crp, *cre;                 // [nb][ntracer]
    const double *qpi, *qepri;         // [nb][ntracer] or null (zero)
    const double *mass;                // [ntracer]
    const unsigned char *dis;          // [ntracer] or null
    Schedule sched;
    unsigned *err;
};

// One host-buffer snapshot in flight: the cell-major spectra of tracer chunk
// k, [bounds[k], bounds[k+1]), are uploaded on the context's h2d stream
// (event pipe_up[k]) and, once evolved (events pipe_done_p[k] after the
// proton steps, pipe_done[k] after the electron steps, on the compute
// stream), downloaded into the same host rows on d2h.
struct HostPipe {
    double *crp = nullptr, *cre = nullptr;   // host [ntracer][nb]
    int down_p = 1, down_e = 1;              // species whose rows come back
    std::vector<int> bounds;                 // chunk starts, then ntracer
};

struct ModelParams {
    int species_mask;
    int dpp_model;
    int ttd_brunetti16;
    double t_acc_direct_gyr;
    double mach_limit;
    double psi3;                 // psi^3
    double eta_dpp_cap;
    double nsub_safety;
    int nsub_max;
    int interp_min_steps, interp_max_segments;
    int window_centred;
    double f_eddy, t_off_gyr, t_acc_off_gyr;
};

// The steps-kernel autotuner's record for one species (fused.cu): the
// variant chosen (solver and warps per block, index into the tuner's list)
// and the calibration time of each variant (-1: not run).
struct TuneState {
    int tuned = 0;
    int variant = 0;
    int tracers = 0, steps = 0;
    double ms[CROMA_B200_STEPS_VARIANTS] = {-1.0, -1.0, -1.0, -1.0, -1.0, -1.0, -1.0, -1.0, -1.0};
};

struct Context {
    CromaB200Config cfg{};
    ModelParams mp{};
    int device = 0;
    cudaStream_t stream = nullptr;

    // host copies of the grids (p, dp, E per species; pm1/pp1); grid_given:
    // filled by the caller (reference ABI) instead of from pmin/pmax
    int grid_given = 0;
    std::vector<double> h_p[2], h_dp[2], h_E[2];
    double h_pm1[2] = {0, 0}, h_pp1[2] = {0, 0};
    std::vector<double> h_fqe;        // [nb][nb] transposed [jp][je]
    std::vector<int> h_np_min_qe;
    int *d_np_min_qe = nullptr;       // [nb]

    double *d_tables = nullptr;       // one block holding every grid table
    GridTables gt{};
    IcConsts icc{};

    // IC rows: [2][nb+2], keyed by redshift
    double *d_ic = nullptr;
    double ic_z[2] = {0, 0};
    int ic_valid[2] = {0, 0};
    int ic_slot_curr = 0;
    // pinned staging of the IC outer abscissae: two slots, each reused only
    // after the copy that last read it has completed (its event)
    double *h_ic_stage = nullptr;
    cudaEvent_t ic_stage_ev[2] = {nullptr, nullptr};
    int ic_stage_next = 0;

    // resident state (cell-major [cap][nb])
    int cap = 0, ntracer = 0;
    double *d_crp = nullptr, *d_cre = nullptr;
    double *d_qpi = nullptr, *d_qepri = nullptr;
    double *d_mass = nullptr;
    unsigned char *d_dis = nullptr;
    int has_sources = 0;
    double *d_bg = nullptr;           // [2][8][cap] staging for host backgrounds

    // schedule
    int *d_sched_int = nullptr;
    unsigned char *d_capped = nullptr;
    Schedule sched{};
    void *d_cub_tmp = nullptr;
    size_t cub_tmp_bytes = 0;
    unsigned long long *d_keys = nullptr, *d_keys_alt = nullptr;
    int *d_vals = nullptr, *d_vals_alt = nullptr, *d_seg_aux = nullptr;

    double *d_inje = nullptr;         // electron source per segment (fused workspace)
    double *d_eta_scale = nullptr;    // [cap] Dpp eta-cap scale of the current slot

    // fused-path workspace, per tracer chunk: factored matrices of every
    // segment [2 species][nseg][sets][chunk][3][nb], proton spectra at the
    // segment starts and the electron source per segment [nseg][chunk][nb]
    double *d_fac = nullptr;
    double *d_np_seg = nullptr;
    void *d_segpre = nullptr;         // per-segment scalars [nseg][chunk] (fused.cu)
    unsigned *d_work = nullptr;       // [2] factor-kernel work counters (fused.cu)
    int fused_chunk = 0, fused_nseg = 0, fused_sets = 0;
    double workspace_bytes = 0.0;     // fused workspace cap; 0 = CROMA_B200_WORKSPACE_GB or 24 GB

    // DSA injection
    CromaB200DsaParams dsa{};
    int dsa_set = 0;
    double *d_dsa_p = nullptr;        // [2][nb] DSA-grid momenta at the FP bins
    unsigned *d_dsa_count = nullptr;
    double *d_dsa_stage = nullptr;    // [10][dsa_stage_cap] host shock fields
    int dsa_stage_cap = 0;

    // host-buffer snapshot (croma_b200_snapshot_host): copy streams and
    // per-chunk events, created on first use; pipe is set for one call
    cudaStream_t h2d_stream = nullptr, d2h_stream = nullptr;
    std::vector<cudaEvent_t> pipe_up, pipe_done, pipe_done_p;
    cudaEvent_t pipe_start = nullptr;   // compute stream's earlier work, gating the uploads
    const HostPipe *pipe = nullptr;

    // steps-kernel autotuner, per species
    TuneState tune[2];

    // resident emission tables (croma_b200_emission_setup)
    EmissionState *emission = nullptr;

    unsigned *d_err = nullptr;
    int last_launches = 0;
    int last_nsub_max = 0;

    // optional per-kernel timing (CUDA events on the context stream)
    int timing = 0;
    struct TimedLaunch { int kind; cudaEvent_t start, stop; };
    std::vector<TimedLaunch> timed;           // recorded, not yet read
    std::vector<cudaEvent_t> event_pool;
    double kernel_ms[4] = {0, 0, 0, 0};
    long long kernel_launches[4] = {0, 0, 0, 0};
};

// Kernel kinds for the timing hooks.
enum KernelKind { kKindEvolve = 0, kKindCoeff = 1, kKindSecondary = 2, kKindSchedule = 3 };
cudaEvent_t pooled_event(Context &ctx);
void timed_begin(Context &ctx, int kind, cudaEvent_t *start);
void timed_end(Context &ctx, int kind, cudaEvent_t start);

// Stream-ordered device memory of a context (cudaMallocAsync / cudaFreeAsync
// on its stream): allocating and freeing never synchronise the device, so
// contexts that run side by side (the request server) do not wait on each
// other's queued work.  Freed blocks stay in the device's pool for the next
// allocation.  Other streams use the memory only after an event recorded on
// the context stream, and host copies go through the context stream too.
cudaError_t dev_alloc_bytes(Context &c, void **p, size_t bytes);
template <class T>
inline cudaError_t dev_alloc(Context &c, T **p, size_t bytes)
{
    return dev_alloc_bytes(c, reinterpret_cast<void **>(p), bytes);
}
void dev_free(Context &c, void *p);
// Page-locked host staging rows for the IC outer abscissae, reused across
// contexts (freeing page-locked memory synchronises the device).
double *acquire_ic_stage();
void release_ic_stage(double *p);

// Error reporting shared by the translation units.
void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
#define CROMA_CUDA(call)                                              \
    do {                                                              \
        cudaError_t e__ = (call);                                     \
        if (e__ != cudaSuccess) return ::croma::cuda_fail(e__, #call); \
    } while (0)

// tables.cu
int build_tables(Context &ctx);
void free_ic_stage(Context &ctx);
int ic_rows(Context &ctx, double z, double *d_out);
// schedule.cu
int schedule_reserve(Context &ctx, int cap);
int run_schedule(Context &ctx, const SnapArgs &a);
// fused.cu: both paths (the plain one as per-step kernels, one slot at a time)
int fused_reserve(Context &ctx, int cap);
// device bytes fused_reserve allocates for cap tracers under a workspace cap
// on path CROMA_PATH_*
double fused_workspace_bytes(const ModelParams &mp, int cap, double workspace_cap, int path);
int run_fused(Context &ctx, const SnapArgs &a);
// the autotuner's choice for a species: solver (0 scan, 1 FP32-refined scan,
// 2 PCR, 3 scan with its constants in shared memory) and warps per block;
// returns 1 once tuned
int tuning_info(const Context &ctx, int species, int *solver, int *wpb);
// dsa.cu
int set_dsa(Context &ctx, const CromaB200DsaParams *prm);
int dsa_inject(Context &ctx, const CromaB200Shocks *sh, double density_unit, double dt_gyr, int mode,
               int reacc_mode, int *ninjected);
void free_dsa(Context &ctx);
// emission.cu
int emission_setup(Context &c, const CromaB200EmissionSetup *s);
int emission_run(Context &c, const double *bg_dev, double z, double *eps_syn, double *eps_ic, double *eps_gamma,
                 double *eps_nu);
int emission_tables(Context &c, int which, double *out);
const CromaB200EmissionSetup &emission_config(const Context &c);
// a device block of at least `bytes` for step outputs, kept by the emission state
cudaError_t emission_out_block(Context &c, size_t bytes, double **out);
// kernels one emission_run call launches for the requested kinds
int emission_launches(const Context &c, bool syn, bool ic, bool gamma, bool nu);
void free_emission(Context &c);

}  // namespace croma
