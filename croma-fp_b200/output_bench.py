"""Output files written from device-resident spectra while the snapshots run.

The batching workload (65,536 tracers, electron + proton, 256 bins, ASA,
nsub <= 500) advances `--snapshots` snapshots twice: once without output,
once writing the CRE and CRP tile slabs of every snapshot straight from the
device state (croma_b200_output_write_state: staging on the context stream,
copy stream, writer thread), flushed and fsync'ed at the end.  Reported: the
wall time per snapshot of both loops, the bytes written, and how much of the
write time the snapshots hid.

    python croma-fp_b200/output_bench.py [--tracers 65536] [--snapshots 6] [--dir /tmp/croma_out]
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import sys
import time

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


def run(ntracer=65536, nsnap=6, directory="/tmp/croma_out", seed=5):
    _package()
    import numpy as np
    import torch
    from croma_fp_b200 import config, native, output, synth
    cfg = config.config1()
    w = synth.Workload(cfg, ntracer, 100, seed=seed)
    fp = native.TracerFP(cfg, path="fused")
    gp, ge = fp.grid(0), fp.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), ntracer, cfg.species)
    bgs = [torch.from_numpy(w.background(30 + k)).cuda() for k in range(nsnap + 2)]

    def loop(outs):
        fp.set_state(crp, cre, mass=w.mass)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(nsnap):
            i = 30 + k
            fp.snapshot(bgs[k].data_ptr(), bgs[k + 1].data_ptr(), float(w.z[i]), float(w.z[i + 1]), True,
                        float(w.dt[i]), float(w.elapsed[i]), sync=False)
            if outs:
                output.OutputFile.write_state(fp, outs[0], outs[1], k + 1)
        fp.sync()
        t_compute = time.perf_counter() - t0
        for o in outs:
            o.close()
        return t_compute, time.perf_counter() - t0

    loop([])                                   # warm-up
    base, _ = loop([])
    shutil.rmtree(directory, ignore_errors=True)
    os.makedirs(directory)
    outs = [output.OutputFile(cfg.nb, directory, "CRE", 0, "tile", nsnap + 1, ntracer, cfg.nb),
            output.OutputFile(cfg.nb, directory, "CRP", 0, "tile", nsnap + 1, ntracer, cfg.nb)]
    t_compute, t_total = loop(outs)
    nbytes = 2 * nsnap * ntracer * cfg.nb * 8
    fp.close()
    shutil.rmtree(directory, ignore_errors=True)
    return {"metric": "snapshot wall time with CR tile output written from device state",
            "tracers": ntracer, "snapshots": nsnap, "bins_per_species": cfg.nb,
            "ms_per_snapshot_no_output": base / nsnap * 1e3,
            "ms_per_snapshot_with_output_queued": t_compute / nsnap * 1e3,
            "ms_per_snapshot_with_output_flushed": t_total / nsnap * 1e3,
            "bytes_written": nbytes, "file_write_gbs": nbytes / t_total / 1e9,
            "directory": directory,
            "workload": "batching: electron_proton, 256 bins, ASA, nsub <= 500; CRE + CRP tile slabs "
                        "of every snapshot"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tracers", type=int, default=65536)
    ap.add_argument("--snapshots", type=int, default=6)
    ap.add_argument("--dir", default="/tmp/croma_out")
    args = ap.parse_args()
    print(json.dumps(run(args.tracers, args.snapshots, args.dir)), flush=True)


if __name__ == "__main__":
    main()
