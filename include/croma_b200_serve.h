/*
 * croma_b200_serve.h -- request serving on one B200: many independent tracer
 * runs (chunks of tracers advanced through a number of snapshots) submitted
 * concurrently, admitted against a device-memory budget and run on separate
 * CUDA streams.
 *
 * A request is what the reference's snapshot driver does for one rank's
 * tracers (include/tracer_fp_solve.inc): for each snapshot k of the request
 * the IC rows, schedule, buckets and evolve of croma_b200_snapshot, with
 * backgrounds interpolated between bg[k] and bg[k+1].  Requests are
 * independent; each gets its own context (croma_b200.h) while it runs.
 *
 * Admission: a request needs an estimated number of device bytes (spectra,
 * backgrounds, schedule and evolve workspace for its tracer count).  Queued
 * requests start in submission order while their estimate fits the budget
 * left; a request larger than the whole budget is refused at submission.
 *
 * Scheduling on the device: each running request's stream gets a CUDA stream
 * priority from its size (ntracer x nsnap, log-scaled between 1e3 and 1e7
 * tracer-snapshots; the smallest requests highest), so the blocks of a small
 * request's kernels start ahead of the blocks a large request still has
 * queued, instead of after them.
 *
 * Lifetime: every pointer in a CromaB200Request must stay valid until the
 * request is done, failed or cancelled.  Functions return 0 (or an id >= 1)
 * on success and a negative code on failure (-1 invalid argument, -3 CUDA,
 * -5 over the memory budget); croma_b200_last_error() describes it.
 */
#ifndef CROMA_B200_SERVE_H
#define CROMA_B200_SERVE_H

#include "croma_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CromaB200Server CromaB200Server;

typedef struct {
    CromaB200Config base;            /* model and grids; nb must equal the library's N.
                                        species_mask is taken per request */
    int device;
    double hbm_budget_bytes;         /* admission budget (device bytes) */
    int max_concurrent;              /* requests running at once (one stream each) */
    double workspace_bytes_per_request;   /* evolve workspace cap per request; 0 = 4 GB */
} CromaB200ServeConfig;

typedef struct {
    int ntracer;
    int species_mask;                /* CROMA_SPECIES_* */
    int nsnap;                       /* snapshots to advance */
    const double *bg;                /* host backgrounds: field f of snapshot k, tracer t at
                                        bg[k * bg_snap_stride + f * bg_field_stride + t] */
    long long bg_field_stride;       /* 0 = ntracer */
    long long bg_snap_stride;        /* 0 = 8 * bg_field_stride */
    const double *z;                 /* [nsnap+1] redshifts */
    const double *dt_snap;           /* [nsnap] Gyr */
    double elapsed0_gyr;             /* time at the start of the first snapshot */
    const double *crp_in, *cre_in;   /* [ntracer][nb] host (NULL = zero) */
    const double *mass_msun;         /* [ntracer] host (NULL = 1e7) */
    double *crp_out, *cre_out;       /* [ntracer][nb] host (NULL skips) */
} CromaB200Request;

enum {
    CROMA_REQ_QUEUED = 0,
    CROMA_REQ_RUNNING = 1,
    CROMA_REQ_DONE = 2,
    CROMA_REQ_FAILED = 3,
    CROMA_REQ_CANCELLED = 4
};

int croma_b200_serve_create(const CromaB200ServeConfig *cfg, CromaB200Server **out);

/* Cancels every request (queued ones at once, running ones before their
 * next snapshot), waits for the running ones to stop, frees the server. */
void croma_b200_serve_destroy(CromaB200Server *srv);

/* Estimated device bytes of a request of ntracer tracers. */
double croma_b200_serve_request_bytes(const CromaB200Server *srv, int ntracer);

/* Queues a request; returns its id (>= 1) or a negative code. */
long long croma_b200_serve_submit(CromaB200Server *srv, const CromaB200Request *req);

/* State of a request (CROMA_REQ_*), or -1 for an unknown id. */
int croma_b200_serve_poll(CromaB200Server *srv, long long id);

/* Waits until the request leaves the queued/running states or timeout_s
 * passes (timeout_s < 0: no limit); returns its state. */
int croma_b200_serve_wait(CromaB200Server *srv, long long id, double timeout_s);

/* Cancels a queued request at once, or a running one before its next
 * snapshot; returns 0, or -1 if the request has already finished. */
int croma_b200_serve_cancel(CromaB200Server *srv, long long id);

/* Outcome of a finished request: its return code, latency (submission to
 * completion) and run time (start to completion), in seconds.  msg (may be
 * NULL) receives the error text of a failed request, up to msg_len bytes. */
int croma_b200_serve_result(CromaB200Server *srv, long long id, int *rc, double *latency_s,
                            double *run_s, char *msg, int msg_len);

/* Queue state and latency percentiles of the requests completed so far. */
int croma_b200_serve_stats(CromaB200Server *srv, int *nqueued, int *nrunning, double *bytes_in_use,
                           int *ncompleted, double *p50_s, double *p99_s);

#ifdef __cplusplus
}
#endif
#endif
