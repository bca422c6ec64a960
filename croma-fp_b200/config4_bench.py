"""Full-pipeline workload at scale: 4,194,304 tracers, electron + proton with
pp secondaries, 512 bins per species, ASA reacceleration, nsub <= 500, and
DSA injection (tracer_state mode) on 5 % of tracer-snapshots (Bernoulli per
tracer-snapshot, Mach U[2, 5]) before every snapshot, on one GPU.

The spectra (4 arrays x 4.2 M x 512 doubles = 69 GB) stay resident; the
evolve workspace runs the tracers in chunks.  Every tracer starts from the
seed spectra; backgrounds and shocks are seeded per snapshot.  Device time
(CUDA events) of DSA + snapshot is reported as tracer-snapshot updates/s.

    python croma-fp_b200/config4_bench.py [--tracers 4194304] [--steps 2] [--warmup 1] [--path fused|plain]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _package():
    if "croma_fp_b200" not in sys.modules:
        import importlib.util
        spec = importlib.util.spec_from_file_location("croma_fp_b200", os.path.join(HERE, "__init__.py"),
                                                      submodule_search_locations=[HERE])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["croma_fp_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["croma_fp_b200"]


def run(ntracer=4194304, steps=2, warmup=1, seed=4242, dsa_fraction=0.05, path="fused"):
    _package()
    import torch
    from croma_fp_b200 import config, native, synth
    cfg = config.config4()
    w = synth.Workload(cfg, ntracer, 100, seed=seed)
    fp = native.TracerFP(cfg, path=path)
    gp, ge = fp.grid(0), fp.grid(1)
    crp1, cre1 = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 1, cfg.species)
    fp.set_state_broadcast(ntracer, crp1[0], cre1[0], 1.0e7)
    fp.set_dsa(config.DsaParams())
    stream = torch.cuda.ExternalStream(fp.stream())
    first = 30
    times, injected, dsa_ms = [], [], []
    for k in range(warmup + steps):
        isnap = first + k
        cur, nxt = w.background(isnap), w.background(isnap + 1)
        sh = synth.shocks(cur, isnap, seed, fraction=dsa_fraction)
        d_cur = torch.from_numpy(cur).cuda()
        d_nxt = torch.from_numpy(nxt).cuda()
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        n_inj = fp.dsa_inject(sh, 1.0, float(w.dt[isnap]), "tracer_state")
        e1.record(stream)
        fp.snapshot(d_cur.data_ptr(), d_nxt.data_ptr(), float(w.z[isnap]), float(w.z[isnap + 1]), True,
                    float(w.dt[isnap]), float(w.elapsed[isnap]), sync=False)
        e2.record(stream)
        fp.sync()
        if k >= warmup:
            times.append(e0.elapsed_time(e2))
            dsa_ms.append(e0.elapsed_time(e1))
            injected.append(n_inj)
    sched = fp.schedule()
    fp.close()
    ms = float(np.mean(times))
    return {"metric": "tracer-snapshot updates/s (DSA + snapshot, device time)",
            "value": ntracer / (ms / 1e3), "ms_per_snapshot": ms, "dsa_ms_per_snapshot": float(np.mean(dsa_ms)),
            "tracers": ntracer, "bins_per_species": 512, "steps": steps, "warmup": warmup, "path": path,
            "dsa_injected_per_snapshot": float(np.mean(injected)),
            "nsub": {"min": int(sched["nsub"].min()), "mean": float(sched["nsub"].mean()),
                     "max": int(sched["nsub"].max())},
            "workload": "electron_proton + pp secondaries, 512 bins, ASA, nsub <= 500, DSA tracer_state "
                        "on 5 % of tracer-snapshots (Mach U[2,5])"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tracers", type=int, default=4194304)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--path", default="fused", choices=["fused", "plain"])
    args = ap.parse_args()
    t0 = time.time()
    res = run(args.tracers, args.steps, args.warmup, path=args.path)
    res["wall_s"] = time.time() - t0
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
