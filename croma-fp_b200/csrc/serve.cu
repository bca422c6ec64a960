// serve.cu -- request serving: a FIFO of independent tracer runs admitted
// against a device-memory budget, run by a pool of host threads, each request
// on its own context (and so its own CUDA stream).  Requests share the GPU;
// their kernels overlap where the streams allow.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "../../include/croma_b200_serve.h"
#include "croma_ctx.cuh"

namespace croma {
namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Req {
    long long id = 0;
    CromaB200Request r{};
    double bytes = 0.0;
    int state = CROMA_REQ_QUEUED;
    bool cancel = false;
    int rc = 0;
    std::string msg;
    double t_submit = 0.0, t_start = 0.0, t_end = 0.0;
};

}  // namespace
}  // namespace croma

using croma::Req;

struct CromaB200Server {
    CromaB200ServeConfig cfg{};
    croma::ModelParams mp{};          // segment / window shape for the workspace estimate
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Req>> queue;
    std::map<long long, std::shared_ptr<Req>> reqs;
    double in_use = 0.0;
    int running = 0;
    bool stop = false;
    long long next_id = 1;
    std::vector<double> latencies;
    std::vector<std::thread> workers;
};

namespace croma {
namespace {

constexpr double kDefaultWorkspace = 4.0e9;

double request_bytes(const CromaB200Server &s, int n)
{
    const double nn = (double)n;
    // spectra and sources (4 x nb doubles), mass, flags, background staging
    // (2 x 8 doubles), schedule, bucket keys and values
    double b = nn * (4.0 * NB * 8 + 8 + 1 + 2 * 8 * 8 + 6 * 4 + 1 + 3 * 8 + 8 * 4);
    const double ws = s.cfg.workspace_bytes_per_request > 0.0 ? s.cfg.workspace_bytes_per_request
                                                              : kDefaultWorkspace;
    b += fused_workspace_bytes(s.mp, n, ws, s.cfg.base.path);
    // grid tables, secondary weights, IC rows, sort scratch, context slack
    b += (double)NB * NB * 8 + 40.0 * NB * 8 + 2.0 * (NB + 2 + 2049) * 8 + 16.0 * nn + 64.0e6;
    return b;
}

int run_request(CromaB200Server &s, Req &q)
{
    const CromaB200Request &r = q.r;
    const int n = r.ntracer;
    CromaB200Config cfg = s.cfg.base;
    cfg.species_mask = r.species_mask;
    CromaB200Context *ctx = nullptr;
    int rc = croma_b200_create(&cfg, s.cfg.device, &ctx);
    if (rc) return rc;
    // smaller requests get higher stream priorities: their kernels' blocks are
    // scheduled ahead of the rest of a large request's grid instead of behind it
    {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess && least != greatest) {
            const double work = (double)n * (double)(r.nsnap > 0 ? r.nsnap : 1);
            double f = (log10(work > 1.0 ? work : 1.0) - 3.0) / 4.0;   // 1e3 .. 1e7 tracer-snapshots
            f = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
            const int prio = greatest + (int)lround(f * (double)(least - greatest));
            rc = croma_b200_set_priority(ctx, prio);
            if (rc) {
                croma_b200_destroy(ctx);
                return rc;
            }
        }
    }
    croma_b200_set_workspace_limit(ctx, s.cfg.workspace_bytes_per_request > 0.0
                                            ? s.cfg.workspace_bytes_per_request
                                            : kDefaultWorkspace);
    std::vector<double> mass;
    if (!r.mass_msun) mass.assign((size_t)n, 1.0e7);
    rc = croma_b200_set_state(ctx, n, r.crp_in, r.cre_in, nullptr, nullptr,
                              r.mass_msun ? r.mass_msun : mass.data(), nullptr);
    const long long fs = r.bg_field_stride > 0 ? r.bg_field_stride : n;
    const long long ss = r.bg_snap_stride > 0 ? r.bg_snap_stride : kNbg * fs;
    const bool packed = fs == n && ss == (long long)kNbg * n;
    std::vector<double> stage;
    if (!packed) stage.resize((size_t)2 * kNbg * n);
    double elapsed = r.elapsed0_gyr;
    for (int k = 0; rc == 0 && k < r.nsnap; k++) {
        {
            std::lock_guard<std::mutex> lk(s.mu);
            if (q.cancel) break;
        }
        const double *cur = r.bg + (size_t)k * ss, *nxt = r.bg + (size_t)(k + 1) * ss;
        if (!packed) {
            for (int f = 0; f < kNbg; f++) {
                memcpy(stage.data() + (size_t)f * n, cur + (size_t)f * fs, (size_t)n * sizeof(double));
                memcpy(stage.data() + (size_t)(kNbg + f) * n, nxt + (size_t)f * fs, (size_t)n * sizeof(double));
            }
            cur = stage.data();
            nxt = stage.data() + (size_t)kNbg * n;
        }
        CromaB200Snapshot snap{};
        snap.bg_curr = cur;
        snap.bg_next = nxt;
        snap.bg_on_device = 0;
        snap.z_curr = r.z[k];
        snap.z_next = r.z[k + 1];
        snap.allow_interp = 1;
        snap.dt_snap = r.dt_snap[k];
        snap.elapsed_gyr = elapsed;
        elapsed += r.dt_snap[k];
        rc = croma_b200_snapshot(ctx, &snap, 0);
    }
    if (rc == 0) rc = croma_b200_sync(ctx);
    if (rc == 0 && (r.crp_out || r.cre_out)) rc = croma_b200_get_state(ctx, r.crp_out, r.cre_out);
    croma_b200_destroy(ctx);
    return rc;
}

void worker(CromaB200Server *s)
{
    cudaSetDevice(s->cfg.device);
    for (;;) {
        std::shared_ptr<Req> q;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                return s->stop ||
                       (!s->queue.empty() && s->queue.front()->bytes <= s->cfg.hbm_budget_bytes - s->in_use);
            });
            if (s->stop) return;
            q = s->queue.front();
            s->queue.pop_front();
            s->in_use += q->bytes;
            s->running += 1;
            q->state = CROMA_REQ_RUNNING;
            q->t_start = now_s();
            s->cv_work.notify_all();   // the next head may fit as well
        }
        set_error("");
        const int rc = run_request(*s, *q);
        const std::string msg = rc ? std::string(croma_b200_last_error()) : std::string();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->in_use -= q->bytes;
            s->running -= 1;
            q->t_end = now_s();
            q->rc = rc;
            q->msg = msg;
            if (q->cancel && rc == 0) {
                q->state = CROMA_REQ_CANCELLED;
            } else if (rc) {
                q->state = CROMA_REQ_FAILED;
            } else {
                q->state = CROMA_REQ_DONE;
                s->latencies.push_back(q->t_end - q->t_submit);
            }
            s->cv_done.notify_all();
            s->cv_work.notify_all();
        }
    }
}

bool finished(int state)
{
    return state == CROMA_REQ_DONE || state == CROMA_REQ_FAILED || state == CROMA_REQ_CANCELLED;
}

}  // namespace
}  // namespace croma

using namespace croma;

extern "C" {

int croma_b200_serve_create(const CromaB200ServeConfig *cfg, CromaB200Server **out)
{
    if (!cfg || !out) { set_error("null argument"); return -1; }
    if (cfg->base.nb != NB) { set_error("config nb does not match this library's bin count"); return -1; }
    if (!(cfg->hbm_budget_bytes > 0.0)) { set_error("hbm_budget_bytes must be positive"); return -1; }
    if (cfg->max_concurrent < 1 || cfg->max_concurrent > 64) {
        set_error("max_concurrent must be in 1..64");
        return -1;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
        set_error("device index out of range");
        return -1;
    }
    auto *s = new (std::nothrow) CromaB200Server();
    if (!s) { set_error("host allocation failed"); return -4; }
    s->cfg = *cfg;
    s->mp.interp_max_segments = cfg->base.coeff_interp_max_segments;
    s->mp.window_centred = cfg->base.reacc_window_mode == 1;
    for (int i = 0; i < cfg->max_concurrent; i++) s->workers.emplace_back(worker, s);
    *out = s;
    return 0;
}

void croma_b200_serve_destroy(CromaB200Server *s)
{
    if (!s) return;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        for (auto &q : s->queue) {
            q->state = CROMA_REQ_CANCELLED;
            q->cancel = true;
        }
        s->queue.clear();
        for (auto &kv : s->reqs) kv.second->cancel = true;
        s->cv_done.wait(lk, [&] { return s->running == 0; });
        s->stop = true;
        s->cv_work.notify_all();
    }
    for (auto &t : s->workers) t.join();
    delete s;
}

double croma_b200_serve_request_bytes(const CromaB200Server *s, int ntracer)
{
    if (!s || ntracer <= 0) return 0.0;
    return request_bytes(*s, ntracer);
}

long long croma_b200_serve_submit(CromaB200Server *s, const CromaB200Request *r)
{
    if (!s || !r) { set_error("null argument"); return -1; }
    if (r->ntracer <= 0 || r->nsnap <= 0 || !r->bg || !r->z || !r->dt_snap) {
        set_error("request needs ntracer > 0, nsnap > 0, backgrounds, redshifts and dt");
        return -1;
    }
    if ((r->species_mask & 3) == 0) { set_error("empty species mask"); return -1; }
    for (int k = 0; k < r->nsnap; k++)
        if (!(r->dt_snap[k] > 0.0)) { set_error("dt_snap must be positive"); return -1; }
    auto q = std::make_shared<Req>();
    q->r = *r;
    q->bytes = request_bytes(*s, r->ntracer);
    if (q->bytes > s->cfg.hbm_budget_bytes) {
        set_error("request exceeds the server's device-memory budget");
        return -5;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) { set_error("server is stopping"); return -1; }
    q->id = s->next_id++;
    q->t_submit = now_s();
    s->reqs[q->id] = q;
    s->queue.push_back(q);
    s->cv_work.notify_all();
    return q->id;
}

int croma_b200_serve_poll(CromaB200Server *s, long long id)
{
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    return it == s->reqs.end() ? -1 : it->second->state;
}

int croma_b200_serve_wait(CromaB200Server *s, long long id, double timeout_s)
{
    if (!s) return -1;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return -1;
    std::shared_ptr<Req> q = it->second;
    auto done = [&] { return finished(q->state); };
    if (timeout_s < 0.0) s->cv_done.wait(lk, done);
    else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    return q->state;
}

int croma_b200_serve_cancel(CromaB200Server *s, long long id)
{
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end() || finished(it->second->state)) return -1;
    std::shared_ptr<Req> q = it->second;
    q->cancel = true;
    if (q->state == CROMA_REQ_QUEUED) {
        s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), q), s->queue.end());
        q->state = CROMA_REQ_CANCELLED;
        q->t_end = now_s();
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
    return 0;
}

int croma_b200_serve_result(CromaB200Server *s, long long id, int *rc, double *latency_s, double *run_s,
                            char *msg, int msg_len)
{
    if (!s) { set_error("null server"); return -1; }
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) { set_error("unknown request id"); return -1; }
    const Req &q = *it->second;
    if (!finished(q.state)) { set_error("request has not finished"); return -1; }
    if (rc) *rc = q.rc;
    if (latency_s) *latency_s = q.t_end - q.t_submit;
    if (run_s) *run_s = q.t_start > 0.0 ? q.t_end - q.t_start : 0.0;
    if (msg && msg_len > 0) {
        strncpy(msg, q.msg.c_str(), (size_t)msg_len - 1);
        msg[msg_len - 1] = '\0';
    }
    return 0;
}

int croma_b200_serve_stats(CromaB200Server *s, int *nqueued, int *nrunning, double *bytes_in_use,
                           int *ncompleted, double *p50_s, double *p99_s)
{
    if (!s) { set_error("null server"); return -1; }
    std::vector<double> lat;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (nqueued) *nqueued = (int)s->queue.size();
        if (nrunning) *nrunning = s->running;
        if (bytes_in_use) *bytes_in_use = s->in_use;
        lat = s->latencies;
    }
    if (ncompleted) *ncompleted = (int)lat.size();
    std::sort(lat.begin(), lat.end());
    // nearest rank
    auto pct = [&](double p) {
        if (lat.empty()) return 0.0;
        size_t k = (size_t)std::ceil(p * (double)lat.size());
        if (k < 1) k = 1;
        return lat[k - 1];
    };
    if (p50_s) *p50_s = pct(0.50);
    if (p99_s) *p99_s = pct(0.99);
    return 0;
}

}  // extern "C"
