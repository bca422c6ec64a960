"""Emission entry points of the reference ABI at tracer-batch scale.

Times the per-snapshot emission calls CROMA makes through
include/fp_cuda_backend.h on 65,536 cells of 256-bin spectra: inverse Compton
(prepare_ic_emission_cuda_batch, 20 bands), hadronic gamma and neutrino
(prepare_gamma_emission_cuda_batch, prepare_neutrino_emission_cuda_batch,
20 bands each) and synchrotron through the pitch-kernel table
(prepare_synch_emission_cuda_batch, 8 frequencies, 32 log B rows).  The
contract is the reference's: host arrays in, host arrays out, so each call
copies the spectra to the device and the emissivities back.  Reported per
entry point: the call's own elapsed time (device events around copies and
kernel), the bytes it moves between host and device, and those bytes over
that time.  `resident` times the same integrals through the native
context (croma_b200_emission_ic / _hadronic / _synch) on spectra already on
the device: only the tables, per-cell inputs and emissivities move.  Inputs
are seeded synthetic spectra, backgrounds and kernel tables of the
reference's shapes.

    python croma-fp_b200/emission_bench.py [--cells 65536] [--calls 5]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import sys

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


def run(ncell=65536, calls=5, seed=11):
    _package()
    from croma_fp_b200 import config, native, ref_abi, synth

    cfg = config.config1()
    nb = cfg.nb
    fp = native.TracerFP(cfg, path="fused")
    gp, ge = fp.grid(0), fp.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), ncell, cfg.species)
    w = synth.Workload(cfg, ncell, 100, seed=seed)
    bg = w.background(20)
    rng = np.random.default_rng(seed)
    n_gas = np.ascontiguousarray(bg[0])
    b_dyn = np.ascontiguousarray(bg[2])
    logb = np.ascontiguousarray(np.log10(b_dyn))
    beta_p = np.ascontiguousarray(gp[0] / np.sqrt(1.0 + gp[0] ** 2))
    nband, nfreq, nlogb = 20, 8, 32
    fic = np.ascontiguousarray(rng.uniform(1e-3, 1.0, (nband, nb)))
    kern = np.ascontiguousarray(rng.uniform(1e-3, 1.0, (nband, nb)))
    table = np.ascontiguousarray(rng.uniform(1e-3, 1.0, (nlogb, nfreq, nb)))

    abi = ref_abi.RefAbi(nb)
    L = abi.lib
    L.prepare_ic_emission_cuda_batch.argtypes = [C.c_void_p] * 4
    cg_p, cg_e = abi.grid(*gp), abi.grid(*ge)
    spec_bytes = ncell * nb * 8

    def timed(name, call, bytes_moved):
        ms = C.c_double()
        if call(C.byref(ms)) != 0:
            raise RuntimeError(f"{name}: {abi.error()}")
        t = []
        for _ in range(calls):
            if call(C.byref(ms)) != 0:
                raise RuntimeError(f"{name}: {abi.error()}")
            t.append(ms.value)
        med = statistics.median(t)
        return {"ms_per_call": round(med, 3), "host_device_bytes": bytes_moved,
                "gbs": round(bytes_moved / (med / 1e3) / 1e9, 1),
                "cells_per_s": round(ncell / (med / 1e3))}

    res = {}
    out_ic = np.empty((ncell, nband))
    ic = ref_abi.FpIcEmissionBatchInput(ncell, nband, 0.1, 8.0, 20.0, ref_abi.dptr(cre), ref_abi.dptr(fic))
    res["ic"] = timed("ic", lambda ms: L.prepare_ic_emission_cuda_batch(
        C.byref(ic), C.byref(cg_e), ref_abi.dptr(out_ic), ms), spec_bytes + fic.nbytes + out_ic.nbytes)

    out_h = np.empty((ncell, nband))
    had = ref_abi.FpHadronicEmissionBatchInput(ncell, nband, 0.1, -1.0, 3.0, ref_abi.dptr(n_gas),
                                               ref_abi.dptr(crp), ref_abi.dptr(beta_p), ref_abi.dptr(kern))
    hb = spec_bytes + n_gas.nbytes + kern.nbytes + out_h.nbytes
    res["gamma"] = timed("gamma", lambda ms: L.prepare_gamma_emission_cuda_batch(
        C.byref(had), C.byref(cg_p), ref_abi.dptr(out_h), ms), hb)
    res["neutrino"] = timed("neutrino", lambda ms: L.prepare_neutrino_emission_cuda_batch(
        C.byref(had), C.byref(cg_p), ref_abi.dptr(out_h), ms), hb)

    out_s = np.empty((ncell, nfreq))
    sin = ref_abi.FpSynchEmissionBatchInput()
    sin.ncell, sin.nfreq, sin.nlogb = ncell, nfreq, nlogb
    sin.logb_min, sin.inv_dlogb = -9.0, nlogb / 5.0
    sin.pitch_kernel_table = ref_abi.dptr(table)
    sin.b_dyn, sin.logb, sin.cre_batch = ref_abi.dptr(b_dyn), ref_abi.dptr(logb), ref_abi.dptr(cre)
    res["synch_table"] = timed("synch", lambda ms: L.prepare_synch_emission_cuda_batch(
        C.byref(sin), C.byref(cg_e), ref_abi.dptr(out_s), ms),
        spec_bytes + table.nbytes + b_dyn.nbytes + logb.nbytes + out_s.nbytes)

    # the same integrals on spectra already resident in a context
    fp.set_state(crp, cre, mass=w.mass)

    def resident(name, call, bytes_moved):
        call()
        t = [call()[1] for _ in range(calls)]
        med = statistics.median(t)
        return {"ms_per_call": round(med, 3), "host_device_bytes": bytes_moved,
                "cells_per_s": round(ncell / (med / 1e3)),
                "speedup_vs_reference_contract": round(res[name]["ms_per_call"] / med, 1)}

    nb_b = ncell * 8
    resident_res = {
        "ic": resident("ic", lambda: fp.emission_ic(fic), fic.nbytes + out_ic.nbytes),
        "gamma": resident("gamma", lambda: fp.emission_hadronic(kern, n_gas, beta_p, -1.0, 3.0),
                          nb_b + beta_p.nbytes + kern.nbytes + out_h.nbytes),
        "synch_table": resident("synch_table", lambda: fp.emission_synch(table, b_dyn, logb, -9.0, nlogb / 5.0),
                                table.nbytes + 2 * nb_b + out_s.nbytes),
    }
    fp.close()
    return {"metric": "emission entry points, host buffers in and out (reference contract)",
            "resident": resident_res,
            "cells": ncell, "bins_per_species": nb, "bands": nband, "synch_frequencies": nfreq,
            "synch_logb_rows": nlogb, "calls": calls, "host_buffers": "pageable (numpy)",
            "data": "synthetic (seeded)", "results": res}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cells", type=int, default=65536)
    ap.add_argument("--calls", type=int, default=5)
    a = ap.parse_args()
    print(json.dumps(run(a.cells, a.calls)), flush=True)


if __name__ == "__main__":
    main()
