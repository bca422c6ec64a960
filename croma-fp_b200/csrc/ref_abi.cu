// ref_abi.cu -- the reference-compatible C ABI (include/fp_cuda_backend.h).
//
// Each entry point keeps the reference's name, arguments, ownership and
// return codes (include/fp_cuda_backend.h:92-159 of kosukenishiwaki/croma-fp)
// and runs on this library's kernels:
//
//   run_tracer_pipeline      one (bucket, segment) call of the snapshot driver
//                            (include/tracer_fp_solve.inc:1341-1463): rows and
//                            factorisation on chip, fused sub-steps (fused.cu),
//                            secondary source of the segment
//   cuda_rank_state_*        rank-global device spectra and sources
//                            (src/fp_cuda_workspace.cu:440-524)
//   solve_cc_cuda_batch      one implicit Chang-Cooper step for a batch of
//                            tridiagonal systems (src/fp_cuda_solver.cu:436-495)
//   prepare_*_emission_cuda_batch
//                            synchrotron (pitch-kernel table), hadronic gamma and
//                            neutrino emissivities (src/fp_cuda_emission.cu)
//
// The workspace builds its grid tables from the first call's CRspectrum grids
// and rebuilds them when the grids change.  Model switches come from CROMA's
// globals when the library is linked into CROMA (weak references) and from
// croma_b200_set_model() otherwise.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <string>
#include <vector>

#define np CROMA_NB
#define npe CROMA_NB
#include "../../include/fp_cuda_backend.h"
#include "croma_segment.cuh"
#include "croma_emission.cuh"

// CROMA's parameter globals (include/params.h): bound when present.
extern "C" {
extern char dpp_mode_spec[] __attribute__((weak));
extern int ttd_tacc_model __attribute__((weak));
extern double t_acc_direct_gyr __attribute__((weak));
extern double eta_dpp_cap __attribute__((weak));
}

using namespace croma;

struct FpCudaPipelineWorkspace {
    Context ctx;
    int ready = 0;
    double key[6] = {0, 0, 0, 0, 0, 0};
    // bucket scratch (capacity bcap tracers)
    int bcap = 0;
    double *b_bg = nullptr;      // [2][8][ncell]
    double *b_ric = nullptr;     // [2][nb][ncell]
    double *b_crp = nullptr, *b_cre = nullptr, *b_qpi = nullptr, *b_qepri = nullptr;   // [ncell][nb]
    double *b_mass = nullptr;
    unsigned char *b_dis = nullptr;
    int *b_idx = nullptr;
    int b_n = 0, b_has_src = 0;
    // rank-global state (capacity rcap tracers)
    int rcap = 0, r_n = 0;
    double *r_crp = nullptr, *r_cre = nullptr, *r_qpi = nullptr, *r_qepri = nullptr;
    std::vector<double> h_stage;   // host staging for field packing
};

namespace {

struct ModelSetter {
    int dpp_model = kDppOff;
    int ttd_model = 1;
    double t_acc_direct = 0.0;
    double eta_cap = 0.0;
};
ModelSetter g_model;
std::mutex g_mutex;

int resolve_dpp_model()
{
    if (&dpp_mode_spec[0] != nullptr) {
        const char *s = dpp_mode_spec;
        if (strcmp(s, "asa") == 0) return kDppAsa;
        if (strcmp(s, "ttd") == 0) return kDppTtd;
        if (strcmp(s, "direct_tacc") == 0 || strcmp(s, "tacc") == 0 || strcmp(s, "direct") == 0)
            return kDppDirect;
        return kDppOff;   // resolve_momentumdiff_model, src/fp_shared_core.c:932-957
    }
    return g_model.dpp_model;
}

void fill_model(ModelParams &mp, double psi, double mach_limit)
{
    mp.species_mask = 3;
    mp.dpp_model = resolve_dpp_model();
    mp.ttd_brunetti16 = (&ttd_tacc_model != nullptr) ? (ttd_tacc_model == 1) : (g_model.ttd_model == 1);
    mp.t_acc_direct_gyr = (&t_acc_direct_gyr != nullptr) ? t_acc_direct_gyr : g_model.t_acc_direct;
    mp.eta_dpp_cap = (&eta_dpp_cap != nullptr) ? eta_dpp_cap : g_model.eta_cap;
    mp.mach_limit = mach_limit;
    mp.psi3 = pow(psi, 3.0);
    mp.t_off_gyr = 0.0;        // the host applies the direct-t_acc schedule per call
    mp.t_acc_off_gyr = 0.0;
    mp.window_centred = 1;
    mp.interp_max_segments = 1;
    mp.interp_min_steps = 1;
}

int fail(int code, const char *msg)
{
    set_error(msg);
    return code;
}

__global__ void gather_rows_kernel(int n, const int *idx, const double *src, double *dst)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (size_t)n * NB) return;
    const int i = (int)(k / NB), j = (int)(k % NB);
    dst[k] = src[(size_t)idx[i] * NB + j];
}

__global__ void scatter_rows_kernel(int n, const int *idx, const double *src, double *dst)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (size_t)n * NB) return;
    const int i = (int)(k / NB), j = (int)(k % NB);
    dst[(size_t)idx[i] * NB + j] = src[k];
}

int ensure_bucket(FpCudaPipelineWorkspace *w, int n)
{
    if (n <= w->bcap) return 0;
    Context &c = w->ctx;
    cudaFree(w->b_bg); cudaFree(w->b_ric); cudaFree(w->b_crp); cudaFree(w->b_cre);
    cudaFree(w->b_qpi); cudaFree(w->b_qepri); cudaFree(w->b_mass); cudaFree(w->b_dis); cudaFree(w->b_idx);
    const size_t st = (size_t)n * NB * sizeof(double);
    CROMA_CUDA(cudaMalloc(&w->b_bg, 2 * (size_t)kNbg * n * sizeof(double)));
    CROMA_CUDA(cudaMalloc(&w->b_ric, 2 * st));
    CROMA_CUDA(cudaMalloc(&w->b_crp, st));
    CROMA_CUDA(cudaMalloc(&w->b_cre, st));
    CROMA_CUDA(cudaMalloc(&w->b_qpi, st));
    CROMA_CUDA(cudaMalloc(&w->b_qepri, st));
    CROMA_CUDA(cudaMalloc(&w->b_mass, (size_t)n * sizeof(double)));
    CROMA_CUDA(cudaMalloc(&w->b_dis, (size_t)n));
    CROMA_CUDA(cudaMalloc(&w->b_idx, (size_t)n * sizeof(int)));
    int rc = fused_reserve(c, n);
    if (rc) return rc;
    w->bcap = n;
    return 0;
}

int ensure_tables(FpCudaPipelineWorkspace *w, const CRspectrum *crp, const CRspectrum *cre)
{
    const double key[6] = {crp->p[0], crp->p[np - 1], crp->pm1, cre->p[0], cre->p[npe - 1], cre->pm1};
    if (w->ready && memcmp(key, w->key, sizeof key) == 0) return 0;
    Context &c = w->ctx;
    c.grid_given = 1;
    const CRspectrum *g[2] = {crp, cre};
    for (int s = 0; s < 2; s++) {
        c.h_p[s].assign(g[s]->p, g[s]->p + NB);
        c.h_dp[s].assign(g[s]->dp, g[s]->dp + NB);
        c.h_E[s].assign(g[s]->E, g[s]->E + NB);
        c.h_pm1[s] = g[s]->pm1;
        c.h_pp1[s] = g[s]->pp1;
    }
    int rc = build_tables(c);
    if (rc) return rc;
    memcpy(w->key, key, sizeof key);
    w->ready = 1;
    return 0;
}

// Upload one FpCoeffBatchInput field set (8 background fields) into a
// field-major [8][n] device block through host staging.
int upload_bg(FpCudaPipelineWorkspace *w, const double *const f[8], int n, double *dst)
{
    w->h_stage.resize((size_t)kNbg * n);
    for (int k = 0; k < kNbg; k++) {
        if (f[k]) memcpy(w->h_stage.data() + (size_t)k * n, f[k], (size_t)n * sizeof(double));
        else memset(w->h_stage.data() + (size_t)k * n, 0, (size_t)n * sizeof(double));
    }
    CROMA_CUDA(cudaMemcpyAsync(dst, w->h_stage.data(), (size_t)kNbg * n * sizeof(double),
                               cudaMemcpyHostToDevice, w->ctx.stream));
    CROMA_CUDA(cudaStreamSynchronize(w->ctx.stream));
    return 0;
}

double elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

// ---- one implicit Chang-Cooper step per system: fp_thomas_solve_ws with the
// RHS of solve_cc_batch_cpu_timed (src/fp_shared_core.c:226-257, 564-615).
// cprime is the kernel's scratch, [nsys][nrow].
__global__ void cc_thomas_kernel(int nsys, int nrow, double dt, const double *a, const double *b,
                                 const double *c, const double *src, const double *x_in,
                                 double *x_out, double *cprime, unsigned *err)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const size_t o = (size_t)s * nrow;
    double *cp = cprime + o;
    double *x = x_out + o;
    if (fabs(b[o]) <= 1.0e-300) { atomicOr(err, kErrSingular); return; }
    cp[0] = -c[o] / b[o];
    x[0] = (dt * src[o] + x_in[o]) / b[o];
    for (int i = 1; i < nrow; i++) {
        const double den = b[o + i] + a[o + i] * cp[i - 1];
        if (fabs(den) <= 1.0e-300) { atomicOr(err, kErrSingular); return; }
        cp[i] = (i == nrow - 1) ? 0.0 : -c[o + i] / den;
        x[i] = ((dt * src[o + i] + x_in[o + i]) + a[o + i] * x[i - 1]) / den;
    }
    for (int i = nrow - 2; i >= 0; i--) x[i] -= cp[i] * x[i + 1];
}

// solve_cc_pcr_kernel's algorithm (src/fp_cuda_solver.cu:144-206): one block
// per system, one thread per row, parallel cyclic reduction over shared
// memory -- at stride s row i absorbs rows i - s and i + s:
// alpha = a_i / b_{i-s}, gamma = c_i / b_{i+s}; b <- b - alpha c_{i-s} -
// gamma a_{i+s}; a <- alpha a_{i-s}; c <- gamma c_{i+s}; d <- d + alpha
// d_{i-s} + gamma d_{i+s} -- for log2(nrow) levels, then x_i = d_i / b_i.
// nrow is a power of two (checked by the caller); smem 8 nrow doubles.
__global__ void cc_pcr_kernel(int nrow, double dt, const double *a, const double *b, const double *c,
                              const double *src, const double *x_in, double *x_out, unsigned *err)
{
    extern __shared__ double pcr_sm[];
    double *A = pcr_sm, *B = A + nrow, *Cc = B + nrow, *D = Cc + nrow;   // current level
    double *A2 = D + nrow, *B2 = A2 + nrow, *C2 = B2 + nrow, *D2 = C2 + nrow;   // next level
    const int i = threadIdx.x;
    const size_t o = (size_t)blockIdx.x * nrow + i;
    A[i] = a[o];
    B[i] = b[o];
    Cc[i] = c[o];
    D[i] = dt * src[o] + x_in[o];
    __syncthreads();
    for (int st = 1; st < nrow; st <<= 1) {
        double na = 0.0, nb = B[i], nc = 0.0, nd = D[i];
        if (i - st >= 0) {
            const double al = A[i] / B[i - st];
            na = al * A[i - st];
            nb -= al * Cc[i - st];
            nd += al * D[i - st];
        }
        if (i + st < nrow) {
            const double ga = Cc[i] / B[i + st];
            nc = ga * Cc[i + st];
            nb -= ga * A[i + st];
            nd += ga * D[i + st];
        }
        A2[i] = na;
        B2[i] = nb;
        C2[i] = nc;
        D2[i] = nd;
        __syncthreads();
        double *t;
        t = A; A = A2; A2 = t;
        t = B; B = B2; B2 = t;
        t = Cc; Cc = C2; C2 = t;
        t = D; D = D2; D2 = t;
    }
    if (fabs(B[i]) <= 1.0e-300) {
        atomicOr(err, kErrSingular);
        x_out[o] = 0.0;
        return;
    }
    x_out[o] = D[i] / B[i];
}

// One-shot device buffers of the stateless entry points (grow-only, guarded).
struct Scratch {
    std::vector<void *> ptrs;
    ~Scratch() { release(); }
    void release()
    {
        for (void *p : ptrs) cudaFree(p);
        ptrs.clear();
    }
    cudaError_t get(void **out, size_t bytes)
    {
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 8);
        if (e == cudaSuccess) ptrs.push_back(p);
        *out = p;
        return e;
    }
};

// Band energies as the reference accumulates them (fp_shared_core.c:2178-2188).
std::vector<double> hadronic_energies(int nbins, double emin, double emax)
{
    std::vector<double> E(nbins);
    const double d = (emax - emin) / (double)nbins;
    double a = emin - d;
    for (int i = 0; i < nbins; i++) {
        a += d;
        E[i] = pow(10.0, a);
    }
    return E;
}

int emission_hadronic(int ncell, int nbins, double emin, double emax, const double *crp_batch,
                      const double *n_gas, const double *beta_p, const double *kern,
                      const CRspectrum *grid, double *out, double *elapsed_ms)
{
    if (ncell <= 0 || nbins <= 0 || !crp_batch || !n_gas || !beta_p || !kern || !grid || !out)
        return fail(-1, "invalid emission arguments");
    const std::vector<double> E = hadronic_energies(nbins, emin, emax);
    Scratch s;
    double *d_crp, *d_n, *d_bp, *d_dp, *d_k, *d_E, *d_out;
    CROMA_CUDA(s.get((void **)&d_crp, (size_t)ncell * NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_n, (size_t)ncell * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_bp, NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_dp, NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_k, (size_t)nbins * NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_E, (size_t)nbins * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_out, (size_t)ncell * nbins * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    CROMA_CUDA(cudaMemcpy(d_crp, crp_batch, (size_t)ncell * NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_n, n_gas, (size_t)ncell * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_bp, beta_p, NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_dp, grid->dp, NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_k, kern, (size_t)nbins * NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_E, E.data(), (size_t)nbins * sizeof(double), cudaMemcpyHostToDevice));
    dim3 blk(32, 4), grd((ncell + 31) / 32, (nbins + 3) / 4);
    hadronic_emission_kernel<<<grd, blk>>>(ncell, nbins, d_crp, d_n, d_bp, d_dp, d_k, d_E, d_out);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpy(out, d_out, (size_t)ncell * nbins * sizeof(double), cudaMemcpyDeviceToHost));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

}  // namespace

extern "C" {

int croma_b200_set_model(int dpp_model, int ttd_model, double t_acc_direct, double eta_cap)
{
    if (dpp_model < 1 || dpp_model > 4) return fail(-1, "unknown dpp model");
    std::lock_guard<std::mutex> lk(g_mutex);
    g_model.dpp_model = dpp_model;
    g_model.ttd_model = ttd_model;
    g_model.t_acc_direct = t_acc_direct;
    g_model.eta_cap = eta_cap;
    return 0;
}

int cuda_pipeline_is_available(void)
{
    int n = 0;
    return (cudaGetDeviceCount(&n) == cudaSuccess && n > 0) ? 1 : 0;
}

int cuda_bind_local_rank(int local_rank, int *device_out)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return fail(-1, "no CUDA device available");
    if (local_rank < 0) return fail(-1, "negative local rank");
    const int dev = local_rank % n;
    CROMA_CUDA(cudaSetDevice(dev));
    if (device_out) *device_out = dev;
    return 0;
}

int cuda_get_binding_state(int *device_count_out, int *current_device_out)
{
    int n = 0, cur = -1;
    if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
    if (n > 0) cudaGetDevice(&cur);
    if (device_count_out) *device_count_out = n;
    if (current_device_out) *current_device_out = cur;
    return n > 0 ? 0 : -1;
}

int cuda_get_current_device_id(char *out, int len)
{
    if (!out || len <= 0) return fail(-1, "invalid buffer");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(-1, "no current device");
    CROMA_CUDA(cudaDeviceGetPCIBusId(out, len, dev));
    return 0;
}

// CROMA_CUDA_TRIDIAG as the reference reads it (src/fp_cuda_solver.cu:41-72):
// "pcr" selects PCR for power-of-two row counts up to 512 (-1 otherwise),
// "thomas" selects Thomas.  Unset, this library's solvers are Thomas (the
// stateless batch solve) and, in the pipeline, the steps-kernel autotuner's
// choice, which has picked the warp-scan Thomas over warp PCR on every
// configuration measured; the stateless query then reports Thomas.
int fp_cuda_tridiag_uses_pcr(int nrow)
{
    const char *e = getenv("CROMA_CUDA_TRIDIAG");
    if (!e) e = getenv("FP_GPU_CUDA_TRIDIAG");
    if (!e || strcmp(e, "pcr") != 0) return 0;
    return (nrow > 0 && (nrow & (nrow - 1)) == 0 && nrow <= 512) ? 1 : -1;
}

const char *fp_cuda_tridiag_solver_name(int nrow)
{
    const int pcr = fp_cuda_tridiag_uses_pcr(nrow);
    if (pcr > 0) return "PCR (parallel cyclic reduction, one block per system)";
    if (pcr < 0) return "PCR requested for a row count it cannot take";
    return "Thomas (warp-scan LU, factor once per segment)";
}

int solve_cc_cuda_batch(const FpChangCooperSolveBatchInput *in, const double *state_init,
                        double *state_out, double *elapsed_ms, int *used_pcr_out)
{
    if (!in || !state_init || !state_out || in->nsys <= 0 || in->nrow <= 1 || !in->a_batch ||
        !in->b_batch || !in->c_batch || !in->source_batch)
        return fail(-1, "invalid solve_cc_cuda_batch arguments");
    const size_t n = (size_t)in->nsys * in->nrow, bytes = n * sizeof(double);
    Scratch s;
    double *d[7];
    for (int k = 0; k < 7; k++) CROMA_CUDA(s.get((void **)&d[k], bytes));
    unsigned *d_err = nullptr;
    CROMA_CUDA(s.get((void **)&d_err, sizeof(unsigned)));
    CROMA_CUDA(cudaMemset(d_err, 0, sizeof(unsigned)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    const double *h[5] = {in->a_batch, in->b_batch, in->c_batch, in->source_batch, state_init};
    for (int k = 0; k < 5; k++) CROMA_CUDA(cudaMemcpy(d[k], h[k], bytes, cudaMemcpyHostToDevice));
    const int pcr = fp_cuda_tridiag_uses_pcr(in->nrow);
    if (pcr < 0) return fail(-1, "CROMA_CUDA_TRIDIAG=pcr needs a power-of-two row count of at most 512");
    if (pcr) {
        cc_pcr_kernel<<<in->nsys, in->nrow, 8 * in->nrow * sizeof(double)>>>(in->nrow, in->dt, d[0], d[1], d[2],
                                                                             d[3], d[4], d[5], d_err);
    } else {
        cc_thomas_kernel<<<(in->nsys + 127) / 128, 128>>>(in->nsys, in->nrow, in->dt, d[0], d[1], d[2], d[3],
                                                          d[4], d[5], d[6], d_err);
    }
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpy(state_out, d[5], bytes, cudaMemcpyDeviceToHost));
    unsigned err = 0;
    CROMA_CUDA(cudaMemcpy(&err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (used_pcr_out) *used_pcr_out = pcr;
    if (err) return fail(-2, "singular tridiagonal pivot in solve_cc_cuda_batch");
    return 0;
}

FpCudaPipelineWorkspace *cuda_pipeline_workspace_create(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        set_error("no CUDA device available");
        return nullptr;
    }
    auto *w = new (std::nothrow) FpCudaPipelineWorkspace();
    if (!w) return nullptr;
    Context &c = w->ctx;
    cudaGetDevice(&c.device);
    c.cfg.nb = NB;
    c.cfg.species_mask = 3;
    c.cfg.path = CROMA_PATH_FUSED;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c.d_err, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(c.d_err, 0, sizeof(unsigned)) != cudaSuccess) {
        set_error("workspace creation failed");
        cuda_pipeline_workspace_destroy(w);
        return nullptr;
    }
    return w;
}

void cuda_pipeline_workspace_destroy(FpCudaPipelineWorkspace *w)
{
    if (!w) return;
    Context &c = w->ctx;
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    cudaFree(w->b_bg); cudaFree(w->b_ric); cudaFree(w->b_crp); cudaFree(w->b_cre);
    cudaFree(w->b_qpi); cudaFree(w->b_qepri); cudaFree(w->b_mass); cudaFree(w->b_dis); cudaFree(w->b_idx);
    cudaFree(w->r_crp); cudaFree(w->r_cre); cudaFree(w->r_qpi); cudaFree(w->r_qepri);
    // buffers the shared context code allocated on the context stream
    dev_free(c, c.d_inje);
    dev_free(c, c.d_eta_scale);
    dev_free(c, c.d_fac);
    dev_free(c, c.d_np_seg);
    dev_free(c, c.d_segpre);
    dev_free(c, c.d_work);
    dev_free(c, c.d_tables);
    dev_free(c, c.d_np_min_qe);
    if (c.stream) cudaStreamSynchronize(c.stream);
    cudaFree(c.d_err);
    for (auto &t : c.timed) { cudaEventDestroy(t.start); cudaEventDestroy(t.stop); }
    for (auto e : c.event_pool) cudaEventDestroy(e);
    if (c.stream) cudaStreamDestroy(c.stream);
    delete w;
}

int cuda_rank_state_upload(FpCudaPipelineWorkspace *w, int ncell, const double *qpi, const double *qepri,
                           const double *crp, const double *cre, double *elapsed_ms)
{
    if (!w || ncell <= 0) return fail(-1, "invalid rank state upload");
    Context &c = w->ctx;
    CROMA_CUDA(cudaSetDevice(c.device));
    const size_t st = (size_t)ncell * NB * sizeof(double);
    if (ncell > w->rcap) {
        cudaFree(w->r_crp); cudaFree(w->r_cre); cudaFree(w->r_qpi); cudaFree(w->r_qepri);
        CROMA_CUDA(cudaMalloc(&w->r_crp, st));
        CROMA_CUDA(cudaMalloc(&w->r_cre, st));
        CROMA_CUDA(cudaMalloc(&w->r_qpi, st));
        CROMA_CUDA(cudaMalloc(&w->r_qepri, st));
        w->rcap = ncell;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c.stream);
    const double *h[4] = {crp, cre, qpi, qepri};
    double *d[4] = {w->r_crp, w->r_cre, w->r_qpi, w->r_qepri};
    for (int k = 0; k < 4; k++) {
        if (h[k]) CROMA_CUDA(cudaMemcpyAsync(d[k], h[k], st, cudaMemcpyHostToDevice, c.stream));
        else CROMA_CUDA(cudaMemsetAsync(d[k], 0, st, c.stream));
    }
    cudaEventRecord(e1, c.stream);
    CROMA_CUDA(cudaEventSynchronize(e1));
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    w->r_n = ncell;
    return 0;
}

int cuda_rank_state_download(FpCudaPipelineWorkspace *w, int ncell, double *crp, double *cre,
                             double *elapsed_ms)
{
    if (!w || ncell <= 0 || ncell > w->r_n) return fail(-1, "invalid rank state download");
    Context &c = w->ctx;
    CROMA_CUDA(cudaSetDevice(c.device));
    const size_t st = (size_t)ncell * NB * sizeof(double);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c.stream);
    if (crp) CROMA_CUDA(cudaMemcpyAsync(crp, w->r_crp, st, cudaMemcpyDeviceToHost, c.stream));
    if (cre) CROMA_CUDA(cudaMemcpyAsync(cre, w->r_cre, st, cudaMemcpyDeviceToHost, c.stream));
    cudaEventRecord(e1, c.stream);
    CROMA_CUDA(cudaEventSynchronize(e1));
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

int run_tracer_pipeline(const FpCudaPipelineInput *in, const FpCudaOutputSchedule *schedule,
                        double *crp_state_out, double *cre_state_out, double *eps_syn_out,
                        double *eps_gamma_out, double *eps_nu_out, FpCudaPipelineTimes *times)
{
    (void)eps_syn_out;
    (void)eps_gamma_out;
    (void)eps_nu_out;
    if (!in || !in->crp_grid || !in->cre_grid || !in->coeff_in || in->ncell <= 0 || in->nstep < 0)
        return fail(-1, "invalid run_tracer_pipeline arguments");
    if (schedule && (schedule->emit_all_steps || schedule->emit_final_only || schedule->nselected_steps > 0))
        return fail(-1, "in-pipeline emission is not supported; use prepare_*_emission_cuda_batch");
    FpCudaPipelineWorkspace *w = in->workspace;
    if (!w) return fail(-1, "run_tracer_pipeline needs a workspace");
    Context &c = w->ctx;
    CROMA_CUDA(cudaSetDevice(c.device));
    const FpCoeffBatchInput *ci = in->coeff_in;
    const int n = in->ncell;
    // the model first: the bucket workspace is sized by it (on/off factor sets)
    fill_model(c.mp, in->psi_value, in->mach_limit_value);
    c.cfg.species_mask = 3;
    int rc = ensure_tables(w, in->crp_grid, in->cre_grid);
    if (!rc) rc = ensure_bucket(w, n);
    if (rc) return rc;
    cudaEvent_t e0, e1, e2, e3;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
    cudaEventRecord(e0, c.stream);

    // ---- spectra and sources of the bucket ----
    const size_t st = (size_t)n * NB * sizeof(double);
    if (in->gather_rank_state) {
        if (!in->rank_state_indices || !w->r_crp) return fail(-1, "rank state gather without state");
        CROMA_CUDA(cudaMemcpyAsync(w->b_idx, in->rank_state_indices, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
        const int blocks = (int)(((size_t)n * NB + 255) / 256);
        gather_rows_kernel<<<blocks, 256, 0, c.stream>>>(n, w->b_idx, w->r_crp, w->b_crp);
        gather_rows_kernel<<<blocks, 256, 0, c.stream>>>(n, w->b_idx, w->r_cre, w->b_cre);
        gather_rows_kernel<<<blocks, 256, 0, c.stream>>>(n, w->b_idx, w->r_qpi, w->b_qpi);
        gather_rows_kernel<<<blocks, 256, 0, c.stream>>>(n, w->b_idx, w->r_qepri, w->b_qepri);
        w->b_has_src = 1;
        w->b_n = n;
    } else if (in->crp_init || in->cre_init) {
        if (in->crp_init) CROMA_CUDA(cudaMemcpyAsync(w->b_crp, in->crp_init, st, cudaMemcpyHostToDevice, c.stream));
        else CROMA_CUDA(cudaMemsetAsync(w->b_crp, 0, st, c.stream));
        if (in->cre_init) CROMA_CUDA(cudaMemcpyAsync(w->b_cre, in->cre_init, st, cudaMemcpyHostToDevice, c.stream));
        else CROMA_CUDA(cudaMemsetAsync(w->b_cre, 0, st, c.stream));
        if (in->qpi_batch) CROMA_CUDA(cudaMemcpyAsync(w->b_qpi, in->qpi_batch, st, cudaMemcpyHostToDevice, c.stream));
        else CROMA_CUDA(cudaMemsetAsync(w->b_qpi, 0, st, c.stream));
        if (in->qepri_batch) CROMA_CUDA(cudaMemcpyAsync(w->b_qepri, in->qepri_batch, st, cudaMemcpyHostToDevice, c.stream));
        else CROMA_CUDA(cudaMemsetAsync(w->b_qepri, 0, st, c.stream));
        w->b_has_src = (in->qpi_batch || in->qepri_batch) ? 1 : 0;
        w->b_n = n;
    } else if (w->b_n != n) {
        return fail(-1, "no bucket state: pass crp_init/cre_init or gather the rank state");
    }

    // ---- background of the segment (device interpolation when requested) ----
    const int interp = ci->device_interp_background ? 1 : 0;
    {
        const double *cur[8] = {ci->n_gas, ci->kbt, ci->b_field, ci->divv_gyr,
                                ci->l_turb_mpc, ci->dv_imc, ci->cs, ci->beta_pl};
        if (!ci->n_gas || !ci->kbt || !ci->b_field || !ci->divv_gyr || !ci->rad_ic_batch)
            return fail(-1, "incomplete coefficient input");
        if ((rc = upload_bg(w, cur, n, w->b_bg))) return rc;
        CROMA_CUDA(cudaMemcpyAsync(w->b_ric, ci->rad_ic_batch, st, cudaMemcpyHostToDevice, c.stream));
        if (interp) {
            const double *nxt[8] = {ci->n_gas_next, ci->kbt_next, ci->b_field_next, ci->divv_gyr_next,
                                    ci->l_turb_mpc_next, ci->dv_imc_next, ci->cs_next, ci->beta_pl_next};
            if ((rc = upload_bg(w, nxt, n, w->b_bg + (size_t)kNbg * n))) return rc;
            if (ci->rad_ic_batch_next)
                CROMA_CUDA(cudaMemcpyAsync(w->b_ric + (size_t)NB * n, ci->rad_ic_batch_next, st,
                                           cudaMemcpyHostToDevice, c.stream));
            else
                CROMA_CUDA(cudaMemcpyAsync(w->b_ric + (size_t)NB * n, w->b_ric, st, cudaMemcpyDeviceToDevice, c.stream));
        }
        if (ci->tracer_mass_msun)
            CROMA_CUDA(cudaMemcpyAsync(w->b_mass, ci->tracer_mass_msun, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        else
            CROMA_CUDA(cudaMemsetAsync(w->b_mass, 0, n * sizeof(double), c.stream));
        if (ci->disable_adiabatic)
            CROMA_CUDA(cudaMemcpyAsync(w->b_dis, ci->disable_adiabatic, n, cudaMemcpyHostToDevice, c.stream));
        else
            CROMA_CUDA(cudaMemsetAsync(w->b_dis, 0, n, c.stream));
    }
    cudaEventRecord(e1, c.stream);

    // ---- coefficients, secondary source and sub-steps ----
    if (in->nstep > 0) {
        SnapArgs a{};
        a.ntracer = n;
        a.bg_curr = w->b_bg;
        a.bg_next = interp ? w->b_bg + (size_t)kNbg * n : w->b_bg;
        a.ic_curr = w->b_ric;
        a.ic_next = interp ? w->b_ric + (size_t)NB * n : w->b_ric;
        a.allow_interp = interp;
        a.dt_snap = in->dt * in->nstep;
        a.elapsed = 0.0;
        a.crp = w->b_crp;
        a.cre = w->b_cre;
        a.qpi = w->b_has_src ? w->b_qpi : nullptr;
        a.qepri = w->b_has_src ? w->b_qepri : nullptr;
        a.mass = w->b_mass;
        a.dis = w->b_dis;
        a.err = c.d_err;
        SegInfo ex{};
        ex.active = 1;
        ex.nsub = in->nstep;
        ex.nseg = interp ? 2 : 1;
        ex.b = 0;
        ex.e = in->nstep;
        ex.steps = in->nstep;
        ex.windowed = in->use_windowed_reacc ? 1 : 0;
        ex.sl = in->on_start_step;
        ex.el = in->on_end_step;
        ex.alpha = interp ? ci->interp_alpha : 0.0;
        ex.dt = in->dt;
        if ((rc = run_fused_segment(c, a, ex, n))) return rc;
    }
    cudaEventRecord(e2, c.stream);

    // ---- outputs ----
    if (in->scatter_rank_state) {
        if (!in->rank_state_indices || !w->r_crp) return fail(-1, "rank state scatter without state");
        if (!in->gather_rank_state)
            CROMA_CUDA(cudaMemcpyAsync(w->b_idx, in->rank_state_indices, n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
        const int blocks = (int)(((size_t)n * NB + 255) / 256);
        scatter_rows_kernel<<<blocks, 256, 0, c.stream>>>(n, w->b_idx, w->b_crp, w->r_crp);
        scatter_rows_kernel<<<blocks, 256, 0, c.stream>>>(n, w->b_idx, w->b_cre, w->r_cre);
    }
    double *crp_out = crp_state_out ? crp_state_out : in->crp_state_out;
    double *cre_out = cre_state_out ? cre_state_out : in->cre_state_out;
    if (crp_out) CROMA_CUDA(cudaMemcpyAsync(crp_out, w->b_crp, st, cudaMemcpyDeviceToHost, c.stream));
    if (cre_out) CROMA_CUDA(cudaMemcpyAsync(cre_out, w->b_cre, st, cudaMemcpyDeviceToHost, c.stream));
    cudaEventRecord(e3, c.stream);
    CROMA_CUDA(cudaEventSynchronize(e3));
    unsigned err = 0;
    CROMA_CUDA(cudaMemcpy(&err, c.d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (times) {
        memset(times, 0, sizeof(*times));
        times->h2d_ms = elapsed(e0, e1);
        times->solve_ms = elapsed(e1, e2);
        times->d2h_ms = elapsed(e2, e3);
        times->total_ms = elapsed(e0, e3);
        // which sub-step solver the steps-kernel autotuner runs for each species
        int solver = 0;
        if (tuning_info(c, 0, &solver, nullptr)) times->used_pcr_proton = solver == 2;
        if (tuning_info(c, 1, &solver, nullptr)) times->used_pcr_electron = solver == 2;
    }
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
    if (err) {
        cudaMemset(c.d_err, 0, sizeof(unsigned));
        return fail(-2, "kernel reported a numerical failure (singular pivot or NaN CC row)");
    }
    return 0;
}

int run_pipeline_cuda(const FpCudaPipelineInput *in, const FpCudaOutputSchedule *schedule,
                      double *crp_state_out, double *cre_state_out, double *eps_syn_out,
                      double *eps_gamma_out, double *eps_nu_out, FpCudaPipelineTimes *times)
{
    return run_tracer_pipeline(in, schedule, crp_state_out, cre_state_out, eps_syn_out, eps_gamma_out,
                               eps_nu_out, times);
}

int run_tracer_pipeline_group(const FpCudaPipelineInput *inputs, int ninput,
                              const FpCudaOutputSchedule *schedule, FpCudaPipelineTimes *times)
{
    if (!inputs || ninput <= 0) return fail(-1, "invalid pipeline group");
    FpCudaPipelineTimes acc{}, one{};
    for (int i = 0; i < ninput; i++) {
        int rc = run_tracer_pipeline(&inputs[i], schedule, inputs[i].crp_state_out, inputs[i].cre_state_out,
                                     inputs[i].eps_syn_out, inputs[i].eps_gamma_out, inputs[i].eps_nu_out, &one);
        if (rc) return rc;
        acc.h2d_ms += one.h2d_ms;
        acc.solve_ms += one.solve_ms;
        acc.d2h_ms += one.d2h_ms;
        acc.total_ms += one.total_ms;
    }
    if (times) *times = acc;
    return 0;
}

int prepare_ic_emission_cuda_batch(const FpIcEmissionBatchInput *in, const CRspectrum *cre_grid,
                                   double *eps_ic_out, double *elapsed_ms)
{
    if (!in || !cre_grid || !eps_ic_out || in->ncell <= 0 || in->nbins <= 0 || !in->cre_batch ||
        !in->fic_flat)
        return fail(-1, "invalid IC emission input");
    const int ncell = in->ncell, nbins = in->nbins;
    Scratch s;
    double *d_cre, *d_fic, *d_dp, *d_out;
    CROMA_CUDA(s.get((void **)&d_cre, (size_t)ncell * NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_fic, (size_t)nbins * NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_dp, NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_out, (size_t)ncell * nbins * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    CROMA_CUDA(cudaMemcpy(d_cre, in->cre_batch, (size_t)ncell * NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_fic, in->fic_flat, (size_t)nbins * NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_dp, cre_grid->dp, NB * sizeof(double), cudaMemcpyHostToDevice));
    dim3 blk(32, 4), grd((ncell + 31) / 32, (nbins + 3) / 4);
    ic_emission_kernel<<<grd, blk>>>(ncell, nbins, d_cre, d_fic, d_dp, d_out);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpy(eps_ic_out, d_out, (size_t)ncell * nbins * sizeof(double), cudaMemcpyDeviceToHost));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

int prepare_gamma_emission_cuda_batch(const FpGammaEmissionBatchInput *in, const CRspectrum *crp_grid,
                                      double *eps_gamma_out, double *elapsed_ms)
{
    if (!in) return fail(-1, "null gamma input");
    return emission_hadronic(in->ncell, in->nbins, in->egamma_min, in->egamma_max, in->crp_batch,
                             in->n_gas, in->beta_p, in->fga_flat, crp_grid, eps_gamma_out, elapsed_ms);
}

int prepare_neutrino_emission_cuda_batch(const FpNeutrinoEmissionBatchInput *in, const CRspectrum *crp_grid,
                                         double *eps_nu_out, double *elapsed_ms)
{
    if (!in) return fail(-1, "null neutrino input");
    return emission_hadronic(in->ncell, in->nbins, in->enu_min, in->enu_max, in->crp_batch,
                             in->n_gas, in->beta_p, in->fnu_flat, crp_grid, eps_nu_out, elapsed_ms);
}

}  // extern "C"

namespace {

int synch_emission_theta(const FpSynchEmissionBatchInput *in, const CRspectrum *cre_grid, double *eps_syn_out,
                         double *elapsed_ms);

// The F(x) table, pitch weights and logy of a synchrotron input on the
// device (logy gathered from the caller's [nfreq][npe][ntheta] pointer view).
struct SynchTables {
    SynchFx F{};
    double *d_logy = nullptr, *d_w = nullptr;
};

int upload_synch_tables(const FpSynchEmissionBatchInput *in, Scratch &s, SynchTables &t)
{
    if (in->nx_tab <= 0 || in->ntheta_pitch <= 0 || !in->fx_tab || !in->logfx_tab || !in->logx_tab ||
        !in->logy || !in->pitch_weight)
        return fail(-1, "incomplete synchrotron tables (fx, logfx, logx, logy, pitch weights)");
    const int nx = in->nx_tab, nth = in->ntheta_pitch, nfreq = in->nfreq;
    std::vector<double> logy((size_t)nfreq * NB * nth);
    for (int nf = 0; nf < nfreq; nf++) {
        if (!in->logy[nf]) return fail(-1, "null logy plane");
        for (int je = 0; je < NB; je++) {
            if (!in->logy[nf][je]) return fail(-1, "null logy row");
            memcpy(logy.data() + ((size_t)nf * NB + je) * nth, in->logy[nf][je], (size_t)nth * sizeof(double));
        }
    }
    double *d_logx = nullptr, *d_logfx = nullptr;
    CROMA_CUDA(s.get((void **)&d_logx, (size_t)nx * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_logfx, (size_t)nx * sizeof(double)));
    CROMA_CUDA(s.get((void **)&t.d_logy, logy.size() * sizeof(double)));
    CROMA_CUDA(s.get((void **)&t.d_w, (size_t)nth * sizeof(double)));
    CROMA_CUDA(cudaMemcpy(d_logx, in->logx_tab, (size_t)nx * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_logfx, in->logfx_tab, (size_t)nx * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(t.d_logy, logy.data(), logy.size() * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(t.d_w, in->pitch_weight, (size_t)nth * sizeof(double), cudaMemcpyHostToDevice));
    t.F.nx = nx;
    t.F.xmin = in->xmin;
    t.F.inv_dlogx = (nx > 1) ? 1.0 / (in->logx_tab[1] - in->logx_tab[0]) : 0.0;
    t.F.logx_last = in->logx_tab[nx - 1];
    t.F.fx_last = in->fx_tab[nx - 1];
    t.F.logx_tab = d_logx;
    t.F.logfx_tab = d_logfx;
    return 0;
}

}  // namespace

extern "C" {

int prepare_synch_pitch_kernel_table_cuda(const FpSynchEmissionBatchInput *in, double *kernel_table,
                                          double *elapsed_ms)
{
    if (!in || !kernel_table || in->nlogb <= 1 || in->nfreq <= 0 || !(in->inv_dlogb > 0.0))
        return fail(-1, "invalid synchrotron pitch-kernel table input");
    Scratch s;
    SynchTables t;
    int rc = upload_synch_tables(in, s, t);
    if (rc) return rc;
    const size_t n = (size_t)in->nlogb * in->nfreq * NB;
    double *d_table = nullptr;
    CROMA_CUDA(s.get((void **)&d_table, n * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long blocks = ((long long)n + 255) / 256;
    if (blocks > 16LL * nsm) blocks = 16LL * nsm;
    synch_pitch_table_kernel<<<(unsigned)blocks, 256>>>(t.F, in->nfreq, in->ntheta_pitch, in->nlogb,
                                                        in->logb_min, in->inv_dlogb, t.d_logy, t.d_w, d_table);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpy(kernel_table, d_table, n * sizeof(double), cudaMemcpyDeviceToHost));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

int prepare_synch_emission_cuda_batch(const FpSynchEmissionBatchInput *in, const CRspectrum *cre_grid,
                                      double *eps_syn_out, double *elapsed_ms)
{
    if (!in || !cre_grid || !eps_syn_out || in->ncell <= 0 || in->nfreq <= 0)
        return fail(-1, "invalid synchrotron input");
    if (!in->b_dyn || !in->logb || !in->cre_batch) return fail(-1, "incomplete synchrotron input");
    if (!in->pitch_kernel_table || in->nlogb <= 1 || !(in->inv_dlogb > 0.0))
        return synch_emission_theta(in, cre_grid, eps_syn_out, elapsed_ms);
    const int ncell = in->ncell, nfreq = in->nfreq, nlogb = in->nlogb;
    Scratch s;
    double *d_tab, *d_b, *d_lb, *d_cre, *d_dp, *d_out;
    const size_t tab = (size_t)nlogb * nfreq * NB;
    CROMA_CUDA(s.get((void **)&d_tab, tab * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_b, ncell * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_lb, ncell * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_cre, (size_t)ncell * NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_dp, NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_out, (size_t)ncell * nfreq * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    CROMA_CUDA(cudaMemcpy(d_tab, in->pitch_kernel_table, tab * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_b, in->b_dyn, ncell * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_lb, in->logb, ncell * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_cre, in->cre_batch, (size_t)ncell * NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_dp, cre_grid->dp, NB * sizeof(double), cudaMemcpyHostToDevice));
    const SynchPrefactor sp = synch_prefactor();
    dim3 blk(32, 4), grd((ncell + 31) / 32, (nfreq + 3) / 4);
    synch_table_kernel<<<grd, blk>>>(ncell, nfreq, nlogb, in->logb_min, in->inv_dlogb, sp.a0, sp.den1, sp.den2,
                                     d_tab, d_b, d_lb, d_cre, d_dp, d_out);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpy(eps_syn_out, d_out, (size_t)ncell * nfreq * sizeof(double), cudaMemcpyDeviceToHost));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

}  // extern "C"

namespace {

// prepare_synch_emission_cell_major's branch without a pitch-kernel table:
// the pitch-angle integral per (frequency, bin) at each cell's log B.
int synch_emission_theta(const FpSynchEmissionBatchInput *in, const CRspectrum *cre_grid, double *eps_syn_out,
                         double *elapsed_ms)
{
    const int ncell = in->ncell, nfreq = in->nfreq;
    Scratch s;
    SynchTables t;
    int rc = upload_synch_tables(in, s, t);
    if (rc) return rc;
    double *d_b, *d_lb, *d_cre, *d_dp, *d_out;
    CROMA_CUDA(s.get((void **)&d_b, ncell * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_lb, ncell * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_cre, (size_t)ncell * NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_dp, NB * sizeof(double)));
    CROMA_CUDA(s.get((void **)&d_out, (size_t)ncell * nfreq * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    CROMA_CUDA(cudaMemcpy(d_b, in->b_dyn, ncell * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_lb, in->logb, ncell * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_cre, in->cre_batch, (size_t)ncell * NB * sizeof(double), cudaMemcpyHostToDevice));
    CROMA_CUDA(cudaMemcpy(d_dp, cre_grid->dp, NB * sizeof(double), cudaMemcpyHostToDevice));
    const SynchPrefactor sp = synch_prefactor();
    const long long warps = (long long)ncell * nfreq;
    synch_theta_kernel<<<(unsigned)((warps + 3) / 4), 128>>>(t.F, ncell, nfreq, in->ntheta_pitch, sp.a0, sp.den1, sp.den2,
                                                            t.d_logy, t.d_w, d_b, d_lb, d_cre, d_dp, d_out);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpy(eps_syn_out, d_out, (size_t)ncell * nfreq * sizeof(double), cudaMemcpyDeviceToHost));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    if (elapsed_ms) *elapsed_ms = elapsed(e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// Emissivities of a native context's resident spectra (include/croma_b200.h).
// The same kernels as the reference-ABI entry points above, reading the
// spectra where the snapshots left them: only the kernel tables and per-cell
// inputs go up and the emissivities come back.

struct CromaB200Context {
    croma::Context impl;
};

namespace {

struct HostIn {
    const void *src;
    size_t bytes;
};

// One emission call on the context stream: uploads ins into one
// stream-ordered device block, launch(inputs, spectra, dp, out, ncell,
// stream), then the [ntracer][ncols] emissivities to out.
template <class Launch>
int ctx_emission(CromaB200Context *h, int species, int ncols, std::initializer_list<HostIn> ins, double *out,
                 double *elapsed_ms, Launch launch)
{
    if (!h || ncols <= 0 || !out) return fail(-1, "invalid emission arguments");
    Context &c = h->impl;
    const double *spec = species ? c.d_cre : c.d_crp;
    if (c.ntracer <= 0 || !spec) return fail(-1, "no resident spectra: call croma_b200_set_state first");
    if (!(c.mp.species_mask & (species ? CROMA_SPECIES_ELECTRON : CROMA_SPECIES_PROTON)))
        return fail(-1, "emission of a species this context does not evolve");
    for (const HostIn &in : ins)
        if (!in.src || in.bytes == 0) return fail(-1, "missing emission input");
    CROMA_CUDA(cudaSetDevice(c.device));
    const int ncell = c.ntracer;
    auto align = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t out_bytes = (size_t)ncell * ncols * sizeof(double);
    size_t total = align(out_bytes);
    for (const HostIn &in : ins) total += align(in.bytes);
    struct Block {
        Context &c;
        void *p = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Block()
        {
            if (p) dev_free(c, p);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } blk{c};
    CROMA_CUDA(dev_alloc_bytes(c, &blk.p, total));
    CROMA_CUDA(cudaEventCreate(&blk.e0));
    CROMA_CUDA(cudaEventCreate(&blk.e1));
    CROMA_CUDA(cudaEventRecord(blk.e0, c.stream));
    char *p = static_cast<char *>(blk.p);
    double *d_out = reinterpret_cast<double *>(p);
    p += align(out_bytes);
    std::vector<const double *> d_in;
    for (const HostIn &in : ins) {
        CROMA_CUDA(cudaMemcpyAsync(p, in.src, in.bytes, cudaMemcpyHostToDevice, c.stream));
        d_in.push_back(reinterpret_cast<const double *>(p));
        p += align(in.bytes);
    }
    launch(d_in, spec, c.gt.s[species].dp, d_out, ncell, c.stream);
    CROMA_CUDA(cudaGetLastError());
    CROMA_CUDA(cudaMemcpyAsync(out, d_out, out_bytes, cudaMemcpyDeviceToHost, c.stream));
    CROMA_CUDA(cudaEventRecord(blk.e1, c.stream));
    CROMA_CUDA(cudaEventSynchronize(blk.e1));
    if (elapsed_ms) *elapsed_ms = elapsed(blk.e0, blk.e1);
    return 0;
}

}  // namespace

extern "C" {

int croma_b200_emission_ic(CromaB200Context *ctx, int nbands, const double *fic, double *eps_out,
                           double *elapsed_ms)
{
    return ctx_emission(ctx, 1, nbands, {{fic, (size_t)nbands * NB * sizeof(double)}}, eps_out, elapsed_ms,
                        [&](const std::vector<const double *> &in, const double *cre, const double *dp,
                            double *out, int ncell, cudaStream_t st) {
                            dim3 blk(32, 4), grd((ncell + 31) / 32, (nbands + 3) / 4);
                            ic_emission_kernel<<<grd, blk, 0, st>>>(ncell, nbands, cre, in[0], dp, out);
                        });
}

int croma_b200_emission_hadronic(CromaB200Context *ctx, int nbins, double e_min, double e_max,
                                 const double *n_gas, const double *beta_p, const double *kernel,
                                 double *eps_out, double *elapsed_ms)
{
    if (!ctx || nbins <= 0) return fail(-1, "invalid emission arguments");
    const std::vector<double> E = hadronic_energies(nbins, e_min, e_max);
    const size_t ncell = (size_t)(ctx->impl.ntracer > 0 ? ctx->impl.ntracer : 0);
    return ctx_emission(ctx, 0, nbins,
                        {{n_gas, ncell * sizeof(double)}, {beta_p, NB * sizeof(double)},
                         {kernel, (size_t)nbins * NB * sizeof(double)}, {E.data(), (size_t)nbins * sizeof(double)}},
                        eps_out, elapsed_ms,
                        [&](const std::vector<const double *> &in, const double *crp, const double *dp,
                            double *out, int nc, cudaStream_t st) {
                            dim3 blk(32, 4), grd((nc + 31) / 32, (nbins + 3) / 4);
                            hadronic_emission_kernel<<<grd, blk, 0, st>>>(nc, nbins, crp, in[0], in[1], dp, in[2],
                                                                           in[3], out);
                        });
}

int croma_b200_emission_synch(CromaB200Context *ctx, int nfreq, int nlogb, double logb_min, double inv_dlogb,
                              const double *table, const double *b_dyn, const double *logb, double *eps_out,
                              double *elapsed_ms)
{
    if (!ctx || nfreq <= 0) return fail(-1, "invalid emission arguments");
    if (nlogb <= 1 || !(inv_dlogb > 0.0)) return fail(-1, "synchrotron emission needs a pitch-kernel table");
    const size_t ncell = (size_t)(ctx->impl.ntracer > 0 ? ctx->impl.ntracer : 0);
    const SynchPrefactor sp = synch_prefactor();
    return ctx_emission(ctx, 1, nfreq,
                        {{table, (size_t)nlogb * nfreq * NB * sizeof(double)}, {b_dyn, ncell * sizeof(double)},
                         {logb, ncell * sizeof(double)}},
                        eps_out, elapsed_ms,
                        [&](const std::vector<const double *> &in, const double *cre, const double *dp,
                            double *out, int nc, cudaStream_t st) {
                            dim3 blk(32, 4), grd((nc + 31) / 32, (nfreq + 3) / 4);
                            synch_table_kernel<<<grd, blk, 0, st>>>(nc, nfreq, nlogb, logb_min, inv_dlogb, sp.a0, sp.den1,
                                                                    sp.den2, in[0], in[1], in[2], cre, dp, out);
                        });
}

}  // extern "C"
