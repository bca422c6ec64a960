// api.cu -- the native C ABI (include/croma_b200.h).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "croma_ctx.cuh"

struct CromaB200Context {
    croma::Context impl;
};

namespace croma {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char *what)
{
    set_error(std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
              ") at " + what);
    return -3;
}

// The device's default pool keeps up to this many freed bytes for reuse
// (instead of returning them to the driver at each synchronisation).
constexpr uint64_t kPoolKeepBytes = 16ull << 30;

cudaError_t dev_alloc_bytes(Context &c, void **p, size_t bytes)
{
    static std::mutex mu;
    static bool configured[64] = {};
    if (c.device >= 0 && c.device < 64) {
        std::lock_guard<std::mutex> lk(mu);
        if (!configured[c.device]) {
            cudaMemPool_t pool = nullptr;
            if (cudaDeviceGetDefaultMemPool(&pool, c.device) == cudaSuccess) {
                uint64_t keep = kPoolKeepBytes;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            configured[c.device] = true;
        }
    }
    *p = nullptr;
    if (bytes == 0) return cudaSuccess;
    return cudaMallocAsync(p, bytes, c.stream);
}

void dev_free(Context &c, void *p)
{
    if (p) cudaFreeAsync(p, c.stream);
}

cudaEvent_t pooled_event(Context &ctx)
{
    cudaEvent_t e = nullptr;
    if (!ctx.event_pool.empty()) {
        e = ctx.event_pool.back();
        ctx.event_pool.pop_back();
        return e;
    }
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

void timed_begin(Context &ctx, int kind, cudaEvent_t *start)
{
    (void)kind;
    *start = nullptr;
    if (!ctx.timing) return;
    *start = pooled_event(ctx);
    if (*start) cudaEventRecord(*start, ctx.stream);
}

void timed_end(Context &ctx, int kind, cudaEvent_t start)
{
    if (!ctx.timing || !start) return;
    cudaEvent_t stop = pooled_event(ctx);
    if (!stop) return;
    cudaEventRecord(stop, ctx.stream);
    ctx.timed.push_back({kind, start, stop});
}

namespace {

void free_state(Context &c)
{
    dev_free(c, c.d_crp); dev_free(c, c.d_cre); dev_free(c, c.d_qpi); dev_free(c, c.d_qepri);
    dev_free(c, c.d_mass); dev_free(c, c.d_dis); dev_free(c, c.d_bg);
    c.d_crp = c.d_cre = c.d_qpi = c.d_qepri = c.d_mass = c.d_bg = nullptr;
    c.d_dis = nullptr;
    dev_free(c, c.d_inje); dev_free(c, c.d_eta_scale);
    c.d_inje = c.d_eta_scale = nullptr;
    dev_free(c, c.d_fac); dev_free(c, c.d_np_seg); dev_free(c, c.d_segpre); dev_free(c, c.d_work);
    c.d_fac = c.d_np_seg = nullptr;
    c.d_segpre = nullptr;
    c.d_work = nullptr;
    c.fused_chunk = c.fused_nseg = c.fused_sets = 0;
    dev_free(c, c.d_sched_int); dev_free(c, c.d_capped); dev_free(c, c.d_cub_tmp);
    dev_free(c, c.d_keys); dev_free(c, c.d_vals);
    c.d_sched_int = nullptr; c.d_capped = nullptr; c.d_cub_tmp = nullptr;
    c.d_keys = nullptr; c.d_vals = nullptr;
    c.cap = c.ntracer = 0;
}

int check_err(Context &c)
{
    unsigned err = 0;
    CROMA_CUDA(cudaMemcpyAsync(&err, c.d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    if (err) {
        char buf[160];
        snprintf(buf, sizeof buf, "kernel reported numerical failure (bits 0x%x: 1 singular pivot, "
                 "2 NaN at the CC boundary, 4 CMB bound iteration)", err);
        set_error(buf);
        CROMA_CUDA(cudaMemsetAsync(c.d_err, 0, sizeof(unsigned), c.stream));
        return -2;
    }
    return 0;
}

// IC row slot for redshift z (computed on demand), returns device pointer.
int ic_slot(Context &c, double z, int avoid_slot, double **out)
{
    for (int k = 0; k < 2; k++)
        if (c.ic_valid[k] && c.ic_z[k] == z) { *out = c.d_ic + (size_t)k * kIcSlotDoubles; return k; }
    const int k = (avoid_slot == 0) ? 1 : 0;
    int rc = ic_rows(c, z, c.d_ic + (size_t)k * kIcSlotDoubles);
    if (rc != 0) return rc < 0 ? rc - 100 : -100;
    c.ic_valid[k] = 1;
    c.ic_z[k] = z;
    *out = c.d_ic + (size_t)k * kIcSlotDoubles;
    c.last_launches += 1;
    return k;
}

}  // namespace
}  // namespace croma

namespace croma {
namespace {
// row[j] into every tracer's bin j; element (t, j) at base + t * ts + j * js
__global__ void broadcast_rows_kernel(int n, const double *row, double *dst, size_t ts, size_t js)
{
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (size_t)n * NB) return;
    const size_t t = k / NB, j = k % NB;
    dst[t * ts + j * js] = row[j];
}
}  // namespace
}  // namespace croma

using namespace croma;

extern "C" {

const char *croma_b200_last_error(void) { return g_last_error.c_str(); }

int croma_b200_nb(void) { return NB; }

int croma_b200_create(const CromaB200Config *cfg, int device, CromaB200Context **out)
{
    if (cfg == nullptr || out == nullptr) { set_error("null argument"); return -1; }
    if (cfg->nb != NB) { set_error("config nb does not match this library's bin count"); return -1; }
    if (cfg->path != CROMA_PATH_PLAIN && cfg->path != CROMA_PATH_FUSED && cfg->path != CROMA_PATH_FUSED_FP32R) {
        set_error("unknown path");
        return -1;
    }
    if (cfg->dpp_model < 1 || cfg->dpp_model > 4) { set_error("unknown dpp_model"); return -1; }
    if ((cfg->species_mask & 3) == 0) { set_error("empty species mask"); return -1; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        set_error("no CUDA device available");
        return -3;
    }
    if (device < 0 || device >= ndev) { set_error("device index out of range"); return -1; }
    CROMA_CUDA(cudaSetDevice(device));
    auto *h = new (std::nothrow) CromaB200Context();
    if (!h) { set_error("host allocation failed"); return -4; }
    Context &c = h->impl;
    c.cfg = *cfg;
    c.device = device;
    ModelParams &mp = c.mp;
    mp.species_mask = cfg->species_mask & 3;
    mp.dpp_model = cfg->dpp_model;
    mp.ttd_brunetti16 = cfg->ttd_tacc_model == 1;
    mp.t_acc_direct_gyr = cfg->t_acc_direct_gyr;
    mp.mach_limit = cfg->mach_limit;
    mp.psi3 = pow(cfg->psi, 3.0);
    mp.eta_dpp_cap = cfg->eta_dpp_cap;
    mp.nsub_safety = cfg->nsub_safety;
    mp.nsub_max = cfg->nsub_max;
    mp.interp_min_steps = cfg->coeff_interp_min_steps;
    mp.interp_max_segments = cfg->coeff_interp_max_segments;
    mp.window_centred = cfg->reacc_window_mode == 1;
    mp.f_eddy = cfg->f_eddy;
    mp.t_off_gyr = cfg->t_off_gyr;
    mp.t_acc_off_gyr = cfg->t_acc_off_gyr;
    int rc = 0;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) rc = -3;
    if (rc == 0 && dev_alloc(c, &c.d_err, sizeof(unsigned)) != cudaSuccess) rc = -3;
    if (rc == 0 && cudaMemsetAsync(c.d_err, 0, sizeof(unsigned), c.stream) != cudaSuccess) rc = -3;
    if (rc == 0 && dev_alloc(c, &c.d_ic, 2 * (size_t)kIcSlotDoubles * sizeof(double)) != cudaSuccess) rc = -3;
    if (rc == 0) rc = build_tables(c);
    if (rc != 0) {
        if (g_last_error.empty()) set_error("context creation failed");
        croma_b200_destroy(h);
        return rc;
    }
    *out = h;
    return 0;
}

void croma_b200_destroy(CromaB200Context *h)
{
    if (!h) return;
    Context &c = h->impl;
    cudaSetDevice(c.device);
    if (c.stream) cudaStreamSynchronize(c.stream);
    free_state(c);
    for (auto &t : c.timed) { cudaEventDestroy(t.start); cudaEventDestroy(t.stop); }
    for (auto e : c.event_pool) cudaEventDestroy(e);
    dev_free(c, c.d_tables);
    dev_free(c, c.d_np_min_qe);
    dev_free(c, c.d_ic);
    dev_free(c, c.d_err);
    free_ic_stage(c);
    free_dsa(c);
    free_emission(c);
    for (auto e : c.pipe_up) cudaEventDestroy(e);
    for (auto e : c.pipe_done) cudaEventDestroy(e);
    for (auto e : c.pipe_done_p) cudaEventDestroy(e);
    if (c.pipe_start) cudaEventDestroy(c.pipe_start);
    if (c.h2d_stream) cudaStreamDestroy(c.h2d_stream);
    if (c.d2h_stream) cudaStreamDestroy(c.d2h_stream);
    if (c.stream) cudaStreamDestroy(c.stream);
    delete h;
}

int croma_b200_set_workspace_limit(CromaB200Context *h, double bytes)
{
    if (!h || bytes < 0.0 || !isfinite(bytes)) { set_error("invalid workspace limit"); return -1; }
    h->impl.workspace_bytes = bytes;
    return 0;
}

int croma_b200_reserve(CromaB200Context *h, int ntracer)
{
    if (!h || ntracer <= 0) { set_error("invalid reserve"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    if (ntracer == c.cap) { c.ntracer = ntracer; return 0; }
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    free_state(c);
    const size_t n = (size_t)ntracer, st = (size_t)NB * n * sizeof(double);
    CROMA_CUDA(dev_alloc(c, &c.d_crp, st));
    CROMA_CUDA(dev_alloc(c, &c.d_cre, st));
    CROMA_CUDA(dev_alloc(c, &c.d_qpi, st));
    CROMA_CUDA(dev_alloc(c, &c.d_qepri, st));
    CROMA_CUDA(dev_alloc(c, &c.d_mass, n * sizeof(double)));
    CROMA_CUDA(dev_alloc(c, &c.d_dis, n));
    CROMA_CUDA(dev_alloc(c, &c.d_bg, 2 * (size_t)kNbg * n * sizeof(double)));
    CROMA_CUDA(cudaMemsetAsync(c.d_crp, 0, st, c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_cre, 0, st, c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_qpi, 0, st, c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_qepri, 0, st, c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_mass, 0, n * sizeof(double), c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_dis, 0, n, c.stream));
    c.cap = ntracer;
    c.ntracer = ntracer;
    c.has_sources = 0;
    int rc = schedule_reserve(c, ntracer);
    if (rc == 0) rc = fused_reserve(c, ntracer);
    if (rc != 0) { free_state(c); return rc; }
    return 0;
}

int croma_b200_set_state(CromaB200Context *h, int ntracer, const double *crp, const double *cre,
                         const double *qpi, const double *qepri, const double *mass,
                         const unsigned char *dis)
{
    if (!h || ntracer <= 0) { set_error("invalid set_state"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    if (ntracer != c.cap) {
        int rc = croma_b200_reserve(h, ntracer);
        if (rc) return rc;
    }
    const size_t st = (size_t)NB * ntracer * sizeof(double);
    int rc = 0;
    auto up = [&](const double *h, double *d) -> int {
        CROMA_CUDA(cudaMemcpyAsync(d, h, st, cudaMemcpyHostToDevice, c.stream));
        return 0;
    };
    if (crp && (rc = up(crp, c.d_crp))) return rc;
    if (cre && (rc = up(cre, c.d_cre))) return rc;
    if (qpi) { if ((rc = up(qpi, c.d_qpi))) return rc; }
    else CROMA_CUDA(cudaMemsetAsync(c.d_qpi, 0, st, c.stream));
    if (qepri) { if ((rc = up(qepri, c.d_qepri))) return rc; }
    else CROMA_CUDA(cudaMemsetAsync(c.d_qepri, 0, st, c.stream));
    c.has_sources = (qpi != nullptr || qepri != nullptr);
    if (mass) CROMA_CUDA(cudaMemcpyAsync(c.d_mass, mass, ntracer * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    if (dis) CROMA_CUDA(cudaMemcpyAsync(c.d_dis, dis, ntracer, cudaMemcpyHostToDevice, c.stream));
    else CROMA_CUDA(cudaMemsetAsync(c.d_dis, 0, ntracer, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    return 0;
}

int croma_b200_set_state_broadcast(CromaB200Context *h, int ntracer, const double *crp_row,
                                   const double *cre_row, double mass_msun)
{
    if (!h || ntracer <= 0 || !crp_row || !cre_row) { set_error("invalid set_state_broadcast"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    if (ntracer != c.cap) {
        int rc = croma_b200_reserve(h, ntracer);
        if (rc) return rc;
    }
    double *d_rows = nullptr;
    CROMA_CUDA(dev_alloc(c, &d_rows, 2 * NB * sizeof(double)));
    cudaError_t e = cudaMemcpyAsync(d_rows, crp_row, NB * sizeof(double), cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_rows + NB, cre_row, NB * sizeof(double), cudaMemcpyHostToDevice, c.stream);
    const size_t ts = (size_t)NB, js = 1;   // cell-major [tracer][nb]
    const size_t total = (size_t)ntracer * NB;
    const unsigned blocks = (unsigned)((total + 255) / 256);
    if (e == cudaSuccess) {
        broadcast_rows_kernel<<<blocks, 256, 0, c.stream>>>(ntracer, d_rows, c.d_crp, ts, js);
        broadcast_rows_kernel<<<blocks, 256, 0, c.stream>>>(ntracer, d_rows + NB, c.d_cre, ts, js);
        e = cudaGetLastError();
    }
    const size_t st = total * sizeof(double);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_qpi, 0, st, c.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_qepri, 0, st, c.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.d_dis, 0, (size_t)ntracer, c.stream);
    if (e == cudaSuccess) {
        std::vector<double> m((size_t)ntracer, mass_msun);
        e = cudaMemcpyAsync(c.d_mass, m.data(), (size_t)ntracer * sizeof(double), cudaMemcpyHostToDevice, c.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    }
    dev_free(c, d_rows);
    if (e != cudaSuccess) return cuda_fail(e, "set_state_broadcast");
    c.has_sources = 0;
    return 0;
}

int croma_b200_get_state(CromaB200Context *h, double *crp, double *cre)
{
    if (!h) { set_error("null context"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    int rc = 0;
    const size_t st = (size_t)NB * c.cap * sizeof(double);
    auto down = [&](const double *d, double *h) -> int {
        CROMA_CUDA(cudaMemcpyAsync(h, d, st, cudaMemcpyDeviceToHost, c.stream));
        return 0;
    };
    if (crp && (rc = down(c.d_crp, crp))) return rc;
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    if (cre && (rc = down(c.d_cre, cre))) return rc;
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    return check_err(c);
}

int croma_b200_get_sources(CromaB200Context *h, double *qpi, double *qepri, unsigned char *dis)
{
    if (!h) { set_error("null context"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    int rc = 0;
    const size_t st = (size_t)NB * c.cap * sizeof(double);
    auto down = [&](const double *d, double *h) -> int {
        CROMA_CUDA(cudaMemcpyAsync(h, d, st, cudaMemcpyDeviceToHost, c.stream));
        return 0;
    };
    if (qpi && (rc = down(c.d_qpi, qpi))) return rc;
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    if (qepri && (rc = down(c.d_qepri, qepri))) return rc;
    if (dis) CROMA_CUDA(cudaMemcpyAsync(dis, c.d_dis, (size_t)c.cap, cudaMemcpyDeviceToHost, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    return check_err(c);
}

}  // extern "C"

namespace croma {
namespace {

int snapshot_impl(Context &c, const CromaB200Snapshot *s, int sync)
{
    if (c.cap <= 0) { set_error("reserve/set_state before snapshot"); return -1; }
    if (!(s->dt_snap > 0.0)) { set_error("dt_snap must be positive"); return -1; }
    CROMA_CUDA(cudaSetDevice(c.device));
    c.last_launches = 0;
    const size_t n = (size_t)c.cap;
    const int allow = s->allow_interp ? 1 : 0;
    const double *bg_curr = s->bg_curr, *bg_next = allow && s->bg_next ? s->bg_next : s->bg_curr;
    if (!s->bg_on_device) {
        CROMA_CUDA(cudaMemcpyAsync(c.d_bg, bg_curr, kNbg * n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        if (bg_next != bg_curr)
            CROMA_CUDA(cudaMemcpyAsync(c.d_bg + kNbg * n, bg_next, kNbg * n * sizeof(double),
                                       cudaMemcpyHostToDevice, c.stream));
        bg_curr = c.d_bg;
        bg_next = (bg_next != s->bg_curr) ? c.d_bg + kNbg * n : c.d_bg;
    }
    double *ic_cur = nullptr, *ic_nxt = nullptr;
    int k_cur = ic_slot(c, s->z_curr, -1, &ic_cur);
    if (k_cur < 0) return -2;
    if (allow) {
        int k_nxt = ic_slot(c, s->z_next, k_cur, &ic_nxt);
        if (k_nxt < 0) return -2;
    } else {
        ic_nxt = ic_cur;
    }
    SnapArgs a;
    a.ntracer = c.cap;
    a.bg_curr = bg_curr;
    a.bg_next = bg_next;
    a.ic_curr = ic_cur;
    a.ic_next = ic_nxt;
    a.allow_interp = allow;
    a.dt_snap = s->dt_snap;
    a.elapsed = s->elapsed_gyr;
    a.crp = c.d_crp;
    a.cre = c.d_cre;
    a.qpi = c.has_sources ? c.d_qpi : nullptr;
    a.qepri = c.has_sources ? c.d_qepri : nullptr;
    a.mass = c.d_mass;
    a.dis = c.d_dis;
    a.sched = c.sched;
    a.err = c.d_err;
    int rc = run_schedule(c, a);
    if (rc) return rc;
    rc = run_fused(c, a);   // both paths; the plain one runs its per-step kernels
    if (rc) return rc;
    if (sync) return check_err(c);
    return 0;
}

// [from, to) appended to the chunk bounds in near-equal pieces of at most
// maxc tracers.
void push_split(std::vector<int> &b, int from, int to, int maxc)
{
    const long long len = (long long)to - from;
    if (len <= 0) return;
    const long long n = (len + maxc - 1) / maxc;
    for (long long i = 1; i <= n; i++) b.push_back(from + (int)(len * i / n));
}

}  // namespace
}  // namespace croma

extern "C" {

int croma_b200_snapshot(CromaB200Context *h, const CromaB200Snapshot *s, int sync)
{
    if (!h || !s || !s->bg_curr) { set_error("invalid snapshot arguments"); return -1; }
    return snapshot_impl(h->impl, s, sync);
}

int croma_b200_snapshot_host(CromaB200Context *h, const CromaB200Snapshot *s, int ntracer, double *crp,
                             double *cre, const double *mass, int chunks)
{
    if (!h || !s || !s->bg_curr || ntracer <= 0 || !crp || !cre) {
        set_error("invalid snapshot_host arguments");
        return -1;
    }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    if (ntracer != c.cap) {
        const int rc = croma_b200_reserve(h, ntracer);
        if (rc) return rc;
    }
    if (c.fused_chunk <= 0) { set_error("fused workspace not reserved"); return -1; }
    HostPipe pipe;
    pipe.crp = crp;
    pipe.cre = cre;
    pipe.down_p = (c.mp.species_mask & CROMA_SPECIES_PROTON) != 0;
    pipe.down_e = (c.mp.species_mask & CROMA_SPECIES_ELECTRON) != 0;
    // chunk bounds: by default an eighth at each end, so that only a small
    // upload precedes the first kernels and a small download follows the
    // last, and the middle in pieces the workspace holds
    pipe.bounds.push_back(0);
    if (chunks > 0) {
        const long long k = chunks < ntracer ? chunks : ntracer;
        int prev = 0;
        for (long long i = 1; i <= k; i++) {
            const int next = (int)((long long)ntracer * i / k);
            push_split(pipe.bounds, prev, next, c.fused_chunk);
            prev = next;
        }
    } else if (ntracer >= 8192) {
        const int edge = ntracer / 8;
        push_split(pipe.bounds, 0, edge, c.fused_chunk);
        push_split(pipe.bounds, edge, ntracer - edge, c.fused_chunk);
        push_split(pipe.bounds, ntracer - edge, ntracer, c.fused_chunk);
    } else {
        push_split(pipe.bounds, 0, ntracer, c.fused_chunk);
    }
    const int nchunk = (int)pipe.bounds.size() - 1;
    if (!c.h2d_stream) CROMA_CUDA(cudaStreamCreateWithFlags(&c.h2d_stream, cudaStreamNonBlocking));
    if (!c.d2h_stream) CROMA_CUDA(cudaStreamCreateWithFlags(&c.d2h_stream, cudaStreamNonBlocking));
    if (!c.pipe_start) CROMA_CUDA(cudaEventCreateWithFlags(&c.pipe_start, cudaEventDisableTiming));
    while ((int)c.pipe_up.size() < nchunk) {
        cudaEvent_t u = nullptr, d = nullptr, dp = nullptr;
        CROMA_CUDA(cudaEventCreateWithFlags(&u, cudaEventDisableTiming));
        c.pipe_up.push_back(u);
        CROMA_CUDA(cudaEventCreateWithFlags(&d, cudaEventDisableTiming));
        c.pipe_done.push_back(d);
        CROMA_CUDA(cudaEventCreateWithFlags(&dp, cudaEventDisableTiming));
        c.pipe_done_p.push_back(dp);
    }
    // the rest of the state as set_state with these arguments leaves it
    const size_t st = (size_t)NB * ntracer * sizeof(double);
    CROMA_CUDA(cudaMemsetAsync(c.d_qpi, 0, st, c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_qepri, 0, st, c.stream));
    c.has_sources = 0;
    if (mass) CROMA_CUDA(cudaMemcpyAsync(c.d_mass, mass, ntracer * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    CROMA_CUDA(cudaMemsetAsync(c.d_dis, 0, ntracer, c.stream));
    // uploads, chunk by chunk, after whatever the compute stream still runs
    CROMA_CUDA(cudaEventRecord(c.pipe_start, c.stream));
    CROMA_CUDA(cudaStreamWaitEvent(c.h2d_stream, c.pipe_start, 0));
    int rc = 0;
    for (int k = 0; k < nchunk && !rc; k++) {
        const size_t off = (size_t)pipe.bounds[k] * NB;
        const size_t bytes = (size_t)(pipe.bounds[k + 1] - pipe.bounds[k]) * NB * sizeof(double);
        cudaError_t e = cudaMemcpyAsync(c.d_crp + off, crp + off, bytes, cudaMemcpyHostToDevice, c.h2d_stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(c.d_cre + off, cre + off, bytes, cudaMemcpyHostToDevice, c.h2d_stream);
        if (e == cudaSuccess) e = cudaEventRecord(c.pipe_up[k], c.h2d_stream);
        if (e != cudaSuccess) rc = cuda_fail(e, "snapshot_host upload");
    }
    if (!rc) {
        c.pipe = &pipe;
        rc = snapshot_impl(c, s, 0);
        c.pipe = nullptr;
    }
    // the host rows stay in use until both copy streams have drained
    const cudaError_t e1 = cudaStreamSynchronize(c.h2d_stream);
    const cudaError_t e2 = cudaStreamSynchronize(c.d2h_stream);
    if (rc) return rc;
    if (e1 != cudaSuccess) return cuda_fail(e1, "snapshot_host uploads");
    if (e2 != cudaSuccess) return cuda_fail(e2, "snapshot_host downloads");
    return check_err(c);
}

int croma_b200_step_host(CromaB200Context *h, const CromaB200Snapshot *s, const CromaB200StepHost *io)
{
    if (!h || !s || !s->bg_curr || !io || s->bg_on_device) {
        set_error("invalid step_host arguments (host backgrounds required)");
        return -1;
    }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    if (c.cap <= 0 || c.ntracer != c.cap) { set_error("set_state or reserve before step_host"); return -1; }
    if (c.fused_chunk <= 0) { set_error("fused workspace not reserved"); return -1; }
    const size_t n = (size_t)c.cap;
    const bool want_emis = io->eps_syn || io->eps_ic || io->eps_gamma || io->eps_nu;
    if (want_emis && !c.emission) { set_error("emission outputs requested without croma_b200_emission_setup"); return -1; }
    if (!c.h2d_stream) CROMA_CUDA(cudaStreamCreateWithFlags(&c.h2d_stream, cudaStreamNonBlocking));
    if (!c.d2h_stream) CROMA_CUDA(cudaStreamCreateWithFlags(&c.d2h_stream, cudaStreamNonBlocking));
    // 1. the snapshot's backgrounds into the staging block (both slots)
    const int allow = s->allow_interp ? 1 : 0;
    CROMA_CUDA(cudaMemcpyAsync(c.d_bg, s->bg_curr, kNbg * n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    const double *bg_next = c.d_bg;
    if (allow && s->bg_next && s->bg_next != s->bg_curr) {
        CROMA_CUDA(cudaMemcpyAsync(c.d_bg + kNbg * n, s->bg_next, kNbg * n * sizeof(double), cudaMemcpyHostToDevice,
                                   c.stream));
        bg_next = c.d_bg + kNbg * n;
    }
    // 2. DSA injection from the host shock fields (synchronous)
    int launches = 0;
    if (io->shocks && io->dsa_mode != CROMA_DSA_OFF) {
        int nin = 0;
        const int rc = dsa_inject(c, io->shocks, io->density_unit, s->dt_snap, io->dsa_mode, io->dsa_reacc, &nin);
        if (rc) return rc;
        launches += c.last_launches;
    }
    // 3. emission of the spectra the snapshot starts from, downloaded on the
    //    copy stream while the evolve runs
    if (want_emis) {
        const CromaB200EmissionSetup &es = emission_config(c);
        double *host[4] = {io->eps_syn, io->eps_ic, io->eps_gamma, io->eps_nu};
        const int cols[4] = {host[0] ? es.nfreq : 0, host[1] ? es.nbins_ic : 0, host[2] ? es.nbins_gamma : 0,
                             host[3] ? es.nbins_nu : 0};
        size_t total = 0;
        for (int k = 0; k < 4; k++) total += n * (size_t)cols[k];
        // the device outputs stay allocated across calls (grow-only), so a
        // step does not map and unmap gigabytes of device memory each time
        double *d_emis = nullptr;
        CROMA_CUDA(emission_out_block(c, (total ? total : 1) * sizeof(double), &d_emis));
        double *dev[4];
        double *q = d_emis;
        for (int k = 0; k < 4; k++) {
            dev[k] = cols[k] ? q : nullptr;
            q += n * (size_t)cols[k];
        }
        const int rc = emission_run(c, c.d_bg, s->z_curr, dev[0], dev[1], dev[2], dev[3]);
        if (rc) return rc;
        launches += emission_launches(c, dev[0] != nullptr, dev[1] != nullptr, dev[2] != nullptr, dev[3] != nullptr);
        if (!c.pipe_start) CROMA_CUDA(cudaEventCreateWithFlags(&c.pipe_start, cudaEventDisableTiming));
        CROMA_CUDA(cudaEventRecord(c.pipe_start, c.stream));
        CROMA_CUDA(cudaStreamWaitEvent(c.d2h_stream, c.pipe_start, 0));
        for (int k = 0; k < 4; k++)
            if (cols[k])
                CROMA_CUDA(cudaMemcpyAsync(host[k], dev[k], n * cols[k] * sizeof(double), cudaMemcpyDeviceToHost,
                                           c.d2h_stream));
    }
    // 4. the evolve; each workspace chunk's rows go back as soon as it is done
    HostPipe pipe;
    pipe.crp = io->crp_out;
    pipe.cre = io->cre_out;
    pipe.down_p = io->crp_out && (c.mp.species_mask & CROMA_SPECIES_PROTON) != 0;
    pipe.down_e = io->cre_out && (c.mp.species_mask & CROMA_SPECIES_ELECTRON) != 0;
    pipe.bounds.push_back(0);
    push_split(pipe.bounds, 0, (int)n, c.fused_chunk);
    const int nchunk = (int)pipe.bounds.size() - 1;
    while ((int)c.pipe_up.size() < nchunk) {
        cudaEvent_t u = nullptr, d = nullptr, dp = nullptr;
        CROMA_CUDA(cudaEventCreateWithFlags(&u, cudaEventDisableTiming));
        c.pipe_up.push_back(u);
        CROMA_CUDA(cudaEventCreateWithFlags(&d, cudaEventDisableTiming));
        c.pipe_done.push_back(d);
        CROMA_CUDA(cudaEventCreateWithFlags(&dp, cudaEventDisableTiming));
        c.pipe_done_p.push_back(dp);
    }
    // nothing to upload: every chunk's gate is already open
    for (int k = 0; k < nchunk; k++) CROMA_CUDA(cudaEventRecord(c.pipe_up[k], c.stream));
    CromaB200Snapshot sd = *s;
    sd.bg_curr = c.d_bg;
    sd.bg_next = bg_next;
    sd.bg_on_device = 1;
    c.pipe = &pipe;
    int rc = snapshot_impl(c, &sd, 0);
    c.pipe = nullptr;
    launches += c.last_launches;
    const cudaError_t e1 = cudaStreamSynchronize(c.stream);
    const cudaError_t e2 = cudaStreamSynchronize(c.d2h_stream);
    c.last_launches = launches;
    if (rc) return rc;
    if (e1 != cudaSuccess) return cuda_fail(e1, "step_host compute");
    if (e2 != cudaSuccess) return cuda_fail(e2, "step_host downloads");
    return check_err(c);
}

int croma_b200_set_dsa(CromaB200Context *h, const CromaB200DsaParams *params)
{
    if (!h) { set_error("null context"); return -1; }
    CROMA_CUDA(cudaSetDevice(h->impl.device));
    return set_dsa(h->impl, params);
}

int croma_b200_dsa_inject(CromaB200Context *h, const CromaB200Shocks *shocks, double density_unit,
                          double dt_gyr, int mode, int reacc_mode, int *ninjected)
{
    if (!h || !shocks) { set_error("null argument"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    c.last_launches = 0;
    int rc = dsa_inject(c, shocks, density_unit, dt_gyr, mode, reacc_mode, ninjected);
    if (rc) return rc;
    return check_err(c);
}

int croma_b200_get_schedule(CromaB200Context *h, int *nsub, int *non, int *target, int *bucket_ids,
                            int *bucket_indices, int *nbuckets)
{
    if (!h) { set_error("null context"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    const size_t n = (size_t)c.cap * sizeof(int);
    if (nsub) CROMA_CUDA(cudaMemcpyAsync(nsub, c.sched.nsub, n, cudaMemcpyDeviceToHost, c.stream));
    if (non) CROMA_CUDA(cudaMemcpyAsync(non, c.sched.non, n, cudaMemcpyDeviceToHost, c.stream));
    if (target) CROMA_CUDA(cudaMemcpyAsync(target, c.sched.target, n, cudaMemcpyDeviceToHost, c.stream));
    if (bucket_ids) CROMA_CUDA(cudaMemcpyAsync(bucket_ids, c.sched.bucket_ids, n, cudaMemcpyDeviceToHost, c.stream));
    if (bucket_indices)
        CROMA_CUDA(cudaMemcpyAsync(bucket_indices, c.sched.bucket_indices, n, cudaMemcpyDeviceToHost, c.stream));
    if (nbuckets) CROMA_CUDA(cudaMemcpyAsync(nbuckets, c.sched.nbuckets, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    return 0;
}

int croma_b200_ic_row(CromaB200Context *h, double z, double *row_m1_p1)
{
    if (!h || !row_m1_p1) { set_error("null argument"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    double *d = nullptr;
    int k = ic_slot(c, z, -1, &d);
    if (k < 0) return -2;
    CROMA_CUDA(cudaMemcpyAsync(row_m1_p1, d, (NB + 2) * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    return 0;
}

int croma_b200_get_grid(CromaB200Context *h, int species, double *out)
{
    if (!h || !out || species < 0 || species > 1) { set_error("invalid argument"); return -1; }
    Context &c = h->impl;
    memcpy(out, c.h_p[species].data(), NB * sizeof(double));
    memcpy(out + NB, c.h_dp[species].data(), NB * sizeof(double));
    memcpy(out + 2 * NB, c.h_E[species].data(), NB * sizeof(double));
    out[3 * NB] = c.h_pm1[species];
    out[3 * NB + 1] = c.h_pp1[species];
    return 0;
}

int croma_b200_get_secondary_kernel(CromaB200Context *h, double *fqe, int *np_min_qe)
{
    if (!h) { set_error("null context"); return -1; }
    Context &c = h->impl;
    if (fqe) memcpy(fqe, c.h_fqe.data(), c.h_fqe.size() * sizeof(double));
    if (np_min_qe) memcpy(np_min_qe, c.h_np_min_qe.data(), c.h_np_min_qe.size() * sizeof(int));
    return 0;
}

void *croma_b200_stream(CromaB200Context *h) { return h ? (void *)h->impl.stream : nullptr; }

int croma_b200_set_priority(CromaB200Context *h, int priority)
{
    if (!h) { set_error("null context"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    int least = 0, greatest = 0;
    CROMA_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    if (priority > least) priority = least;
    if (priority < greatest) priority = greatest;
    // the context's memory was allocated in this stream's order: let it
    // complete before the stream is replaced
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    cudaStream_t s = nullptr;
    CROMA_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, priority));
    cudaStreamDestroy(c.stream);
    c.stream = s;
    return 0;
}

int croma_b200_sync(CromaB200Context *h)
{
    if (!h) { set_error("null context"); return -1; }
    CROMA_CUDA(cudaSetDevice(h->impl.device));
    return check_err(h->impl);
}

int croma_b200_state_device(CromaB200Context *h, double **crp, double **cre)
{
    if (!h) { set_error("null context"); return -1; }
    if (crp) *crp = h->impl.d_crp;
    if (cre) *cre = h->impl.d_cre;
    return 0;
}

int croma_b200_last_launch_count(CromaB200Context *h) { return h ? h->impl.last_launches : 0; }

int croma_b200_set_kernel_timing(CromaB200Context *h, int enable)
{
    if (!h) { set_error("null context"); return -1; }
    h->impl.timing = enable ? 1 : 0;
    return 0;
}

int croma_b200_kernel_stats(CromaB200Context *h, int kind, double *total_ms, long long *launches)
{
    if (!h || kind < 0 || kind > 3) { set_error("invalid argument"); return -1; }
    Context &c = h->impl;
    CROMA_CUDA(cudaSetDevice(c.device));
    CROMA_CUDA(cudaStreamSynchronize(c.stream));
    for (auto &t : c.timed) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, t.start, t.stop) == cudaSuccess) {
            c.kernel_ms[t.kind] += ms;
            c.kernel_launches[t.kind] += 1;
        }
        c.event_pool.push_back(t.start);
        c.event_pool.push_back(t.stop);
    }
    c.timed.clear();
    if (total_ms) *total_ms = c.kernel_ms[kind];
    if (launches) *launches = c.kernel_launches[kind];
    return 0;
}

int croma_b200_reset_kernel_stats(CromaB200Context *h)
{
    if (!h) { set_error("null context"); return -1; }
    Context &c = h->impl;
    double ms;
    croma_b200_kernel_stats(h, 0, &ms, nullptr);
    for (int k = 0; k < 4; k++) { c.kernel_ms[k] = 0.0; c.kernel_launches[k] = 0; }
    return 0;
}

}  // extern "C"

namespace croma_probe {
// 8 independent FMA chains per thread; the result is written so the work is kept.
__global__ void fp64_fma_probe(int iters, double seed, double *out)
{
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = seed + threadIdx.x * 1e-9 + k * 1e-7;
    const double m = 0.999999999, a = 1e-12;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fma(x[k], m, a);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 12345.678) out[blockIdx.x] = s;
}
// rcp_nr (the factor and per-step kernels' reciprocal) or exp_tab (their
// exponential) element-wise.
__global__ void math_probe(int which, long long n, const double *x, double *out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = which == 0 ? croma::rcp_nr(x[i]) : croma::exp_tab(x[i]);
}
}  // namespace croma_probe

extern "C" {

int croma_b200_get_tuning(CromaB200Context *h, int species, int *tuned, int *solver, int *warps_per_block,
                          double *variant_ms)
{
    if (!h || species < 0 || species > 1) { set_error("invalid get_tuning arguments"); return -1; }
    const Context &c = h->impl;
    const int t = tuning_info(c, species, solver, warps_per_block);
    if (tuned) *tuned = t;
    if (variant_ms)
        for (int v = 0; v < CROMA_B200_STEPS_VARIANTS; v++) variant_ms[v] = c.tune[species].ms[v];
    return 0;
}

int croma_b200_host_alloc(size_t bytes, void **out)
{
    if (!out || bytes == 0) { set_error("invalid host_alloc arguments"); return -1; }
    *out = nullptr;
    CROMA_CUDA(cudaHostAlloc(out, bytes, cudaHostAllocPortable));
    return 0;
}

int croma_b200_host_free(void *p)
{
    if (p) CROMA_CUDA(cudaFreeHost(p));
    return 0;
}

static int math_check(int which, long long n, const double *x, double *out)
{
    if (n < 0 || (n > 0 && (!x || !out))) { set_error("invalid math check arguments"); return -1; }
    if (n == 0) return 0;
    double *d = nullptr;
    CROMA_CUDA(cudaMalloc(&d, 2 * (size_t)n * sizeof(double)));
    cudaError_t e = cudaMemcpy(d, x, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const long long blocks = (n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096;
        croma_probe::math_probe<<<(unsigned)blocks, 256>>>(which, n, d, d + n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "math check");
    return 0;
}

int croma_b200_rcp_check(long long n, const double *x, double *out) { return math_check(0, n, x, out); }
int croma_b200_exp_check(long long n, const double *x, double *out) { return math_check(1, n, x, out); }

int croma_b200_fp64_peak(double *tflops)
{
    if (!tflops) { set_error("null argument"); return -1; }
    int dev = 0, nsm = 0;
    CROMA_CUDA(cudaGetDevice(&dev));
    CROMA_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double *out = nullptr;
    CROMA_CUDA(cudaMalloc(&out, (size_t)nsm * 16 * sizeof(double)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = nsm * 16, threads = 256, iters = 4096;
    croma_probe::fp64_fma_probe<<<blocks, threads>>>(64, 1.0, out);   // warm-up
    cudaEventRecord(e0);
    croma_probe::fp64_fma_probe<<<blocks, threads>>>(iters, 1.0, out);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(e, "fp64 probe");
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return 0;
}

}  // extern "C"
