"""Serving workload: Poisson arrivals of independent tracer runs on one GPU.

Each request advances a chunk of tracers through a number of snapshots:
chunk size log-uniform in [64, 65536], 20..200 snapshots, seed species
uniform over electron-only / proton-only / electron+proton, 256 bins, ASA,
nsub <= 500; arrivals are Poisson at a rate chosen for a target offered load
of the device; the server admits requests against a 120 GB device-memory
budget.  Backgrounds come from one seeded pool shared by all requests (each
request reads a strided window of it); every request starts from the seed
spectra.  Reported: p50 / p99 request latency (submission to completion),
throughput in tracer-snapshot updates/s over the whole run.

    python croma-fp_b200/serve_bench.py [--requests 48] [--load 0.7]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
POOL_TRACERS = 65536
POOL_SNAPS = 201
SEEDS = (("electron_only", 2), ("proton_only", 3), ("electron_proton", 3))


def _package():
    if "croma_fp_b200" not in sys.modules:
        import importlib.util
        spec = importlib.util.spec_from_file_location("croma_fp_b200", os.path.join(HERE, "__init__.py"),
                                                      submodule_search_locations=[HERE])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["croma_fp_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["croma_fp_b200"]


def run(nrequests=48, load=0.7, budget_gb=120.0, max_concurrent=4, seed=20261203,
        rate_tracer_snaps_per_s=1.7e6, pool_tracers=POOL_TRACERS, max_chunk=65536, path="fused"):
    """Runs the serving workload; returns a result dict."""
    _package()
    from croma_fp_b200 import config, serve, synth
    rng = np.random.default_rng(seed)
    cfg = config.config1()
    w = synth.Workload(cfg, pool_tracers, POOL_SNAPS, seed=seed)
    pool = np.empty((POOL_SNAPS, 8, pool_tracers))
    for k in range(POOL_SNAPS):
        pool[k] = w.background(k)
    seeds = {}
    gp = gp_e = None
    from croma_fp_b200 import native
    probe = native.TracerFP(cfg, path="fused")
    gp, ge = probe.grid(0), probe.grid(1)
    probe.close()
    for name, _ in SEEDS:
        seeds[name] = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), max_chunk, name)
    # requests
    sizes = np.exp(rng.uniform(np.log(64), np.log(max_chunk), nrequests)).astype(np.int64)
    nsnaps = rng.integers(20, 201, nrequests)
    kinds = rng.integers(0, 3, nrequests)
    work = float(np.sum(sizes * nsnaps))
    mean_service = work / nrequests / rate_tracer_snaps_per_s
    gaps = rng.exponential(mean_service / load, nrequests)
    srv = serve.Server(cfg, hbm_budget_gb=budget_gb, max_concurrent=max_concurrent, path=path)
    flat = pool.reshape(-1)
    ids = []
    t0 = time.perf_counter()
    next_t = t0
    for i in range(nrequests):
        next_t += gaps[i]
        while time.perf_counter() < next_t:
            time.sleep(min(0.002, max(0.0, next_t - time.perf_counter())))
        n, ns = int(sizes[i]), int(nsnaps[i])
        k0 = int(rng.integers(0, POOL_SNAPS - ns))
        t_off = int(rng.integers(0, pool_tracers - n + 1))
        name, mask = SEEDS[int(kinds[i])]
        crp, cre = seeds[name]
        base = k0 * 8 * pool_tracers + t_off
        rid = srv.submit(flat[base:], w.z[k0:k0 + ns + 1], w.dt[k0:k0 + ns], crp[:n], cre[:n],
                         species_mask=mask, elapsed0=float(w.elapsed[k0]), field_stride=pool_tracers,
                         snap_stride=8 * pool_tracers, ntracer=n)
        ids.append(rid)
    states = [srv.wait(rid) for rid in ids]
    t1 = time.perf_counter()
    lat = []
    for rid in ids:
        rc, l, _, msg = srv.result(rid)
        if rc != 0:
            raise RuntimeError(f"request {rid} failed: {msg}")
        lat.append(l)
        srv.forget(rid)
    st = srv.stats()
    srv.close()
    lat = np.sort(np.array(lat))
    def pct(p):
        return float(lat[max(0, int(np.ceil(p * lat.size)) - 1)])
    return {"requests": nrequests, "done": int(sum(s == serve.DONE for s in states)),
            "p50_s": pct(0.5), "p99_s": pct(0.99), "max_s": float(lat[-1]),
            "tracer_snapshots": work, "wall_s": t1 - t0,
            "throughput": work / (t1 - t0), "offered_load": load, "max_concurrent": max_concurrent,
            "hbm_budget_gb": budget_gb, "server_p50_s": st["p50_s"], "server_p99_s": st["p99_s"], "path": path,
            "workload": "Poisson arrivals, chunk log-U[64, 65536], 20..200 snapshots, "
                        "seed species uniform {e, p, e+p}, 256 bins, ASA, nsub <= 500"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--load", type=float, default=0.7)
    ap.add_argument("--concurrent", type=int, default=4)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    args = ap.parse_args()
    res = run(args.requests, args.load, args.budget_gb, args.concurrent)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
