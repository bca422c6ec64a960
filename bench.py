"""Benchmark: tracer-snapshot updates per second of the Fokker-Planck update,
full pipeline.

Workload (one "step" = one snapshot of every tracer on a GPU): 4,194,304
seeded tracers per GPU, electron + proton spectra with 512 momentum bins
each (protons p/(m_p c) in [1e-2, 1e6], electrons in [1e-1, 1e6]) and
hadronic secondary electrons, ASA reacceleration, sub-step cap 500, on the
100-snapshot z = 1 -> 0 timeline; before every snapshot DSA injection
(tracer_state) on 5 % of the tracers (Bernoulli per tracer-snapshot, Mach
U[2, 5]) and the emission of the spectra the snapshot starts from
(synchrotron at 64 frequencies over 10 MHz..10 GHz; IC, hadronic gamma rays
and neutrinos at 64 energies over 1 keV..1 PeV), as the reference's driver
orders them.  The spectra (2 x 512 x 4.2 M doubles = 34 GB) exceed the
126 MB L2 many times over, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W]
    python bench.py --impl reference      # the reference's CPU code, same workload

Prints one JSON line (rank 0).  ``value`` is the device-timed throughput of
the on-chip FP64 path with every input resident in HBM; ``plain`` the
per-step FP64 path (the reference's data contract) on the same steps;
``e2e`` the same steps through croma_b200_step_host with the inputs read from
and every output (emissivities, evolved spectra) written to page-locked host
memory.  ``fp32r`` is the FP32-refined form on the same steps, ``accuracy``
both forms against the reference's own CPU code on the first 4,096 tracers
over 5 snapshots.  ``secondary.config1`` repeats the measurement on the
65,536-tracer, 256-bin batching workload; ``config2`` runs the
1,048,576-tracer precision workload and compares the FP32-refined spectra
with the FP64 ones on every tracer; ``heavy_tail`` runs a workload whose
sub-step counts spread over 12..500; ``real_histories`` evolves real tracer
histories on backgrounds derived on the device.  ``serving`` is the request
server under a Poisson stream.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
NTRACER = 4194304
NSNAP_TIMELINE = 100
FIRST_SNAP = 30
SEED = 20261203
DSA_FRACTION = 0.05
METRIC = "tracer-snapshot updates/s at <=1e-6 rel err vs FP64, chosen vs plain; p50/p99 latency"
UNIT = "tracer-snapshot updates/s"
SHOCK_KEYS = ("mach", "prestemp", "presden", "shock_side_code")
# DRAM bytes (read + write) per tracer of one launch of each kernel, from the
# ncu captures of this workload's kernels at 16,384 tracers
# (profiles/*_full_pipeline_e_p_512.txt: DRAM rate x duration / 16,384).  Every
# tracer moves its own rows, so a launch's traffic is this figure times the
# tracers it processes.  steps: mean of the proton and electron launches;
# plain_steps: the electron launch of one segment slot.
NCU_DRAM_BYTES_PER_TRACER = {"steps": (272.2e3 + 271.0e3) / 2, "plain_steps": 23.7e3}


def load_package():
    if "croma_fp_b200" in sys.modules:
        return sys.modules["croma_fp_b200"]
    pkg_dir = os.path.join(ROOT, "croma-fp_b200")
    spec = importlib.util.spec_from_file_location(
        "croma_fp_b200", os.path.join(pkg_dir, "__init__.py"), submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["croma_fp_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload_config():
    load_package()
    from croma_fp_b200 import config
    return config.config4()


def workload_desc(ntracer):
    return {"workload": "full pipeline: electron_proton with pp secondaries, 512 bins/species, ASA Dpp, "
                        "nsub capped at 500, DSA tracer_state on 5 % of tracer-snapshots (Mach U[2,5]), "
                        "emission per snapshot (synchrotron 64 freq 10 MHz-10 GHz; IC, gamma, neutrino "
                        "64 bins 1 keV-1 PeV), snapshots 30.. of the z=1->0 100-snapshot timeline",
            "tracers_per_gpu": ntracer, "bins_per_species": 512, "species": "electron_proton",
            "dpp_mode": "asa", "nsub_max": 500, "dsa_fraction": DSA_FRACTION, "precision": "fp64",
            "l2_policy": "inputs larger than L2 (34 GB of spectra per GPU)"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle reasons of one GPU while it runs the timed
    region: polled in-process through NVML every few milliseconds (the device
    matched by PCI bus id), else read from an `nvidia-smi -lms 50` child."""

    NVML_POLL_S = 0.005
    NVML_REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
                    ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
                    ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
                    ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, device_index=0):
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self.dev = device_index
        self.proc = None
        self.t = None
        self.nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            try:
                pr = torch.cuda.get_device_properties(device_index)
                bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.nvml = (pynvml, h)
        except Exception:
            self.nvml = None

    def _poll(self):
        pynvml, h = self.nvml
        bits = [(n, getattr(pynvml, c, 0)) for n, c in self.NVML_REASONS]
        while not self._stop.is_set():
            try:
                self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                for n, bit in bits:
                    if bit and (r & bit):
                        self.reasons.add(n)
            except Exception:
                pass
            self._stop.wait(self.NVML_POLL_S)

    def start(self):
        if self.nvml:
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                self.samples.append(float(parts[1]))
                self.max_mhz = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    self.reasons.add(n)

    def stop(self):
        if self.nvml:
            self._stop.set()
            if self.t:
                self.t.join(timeout=5)
            return
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples),
                "source": "nvml" if self.nvml else "nvidia-smi"}



# ---------------------------------------------------------------- inputs
def make_inputs(cfg, nt, snaps, seed, threads=None):
    """Host backgrounds of snapshots snaps[0] .. snaps[-1] + 1 ([8][nt] each)
    and the shock fields of every step, generated in threads."""
    load_package()
    from croma_fp_b200 import synth
    w = synth.Workload(cfg, nt, NSNAP_TIMELINE, seed=seed)
    isn = list(range(snaps[0], snaps[-1] + 2))
    threads = threads or min(16, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(threads) as ex:
        bgs = list(ex.map(w.background, isn))
        shocks = list(ex.map(lambda k: synth.shocks(bgs[k], isn[k], seed, fraction=DSA_FRACTION),
                             range(len(snaps))))
    return w, bgs, shocks


def seed_rows(fp, cfg):
    from croma_fp_b200 import synth
    gp, ge = fp.grid(0), fp.grid(1)
    crp1, cre1 = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 1, cfg.species)
    return crp1[0], cre1[0]


# ---------------------------------------------------------------- one path, device-resident
def run_resident(path, cfg, nt, w, bg_dev, sh_dev, snaps, warmup, steps, emission=True, dsa=True,
                 kernel_timing=False, clock_dev=None, keep_open=False):
    """DSA + emission + snapshot per step on the resident spectra, inputs
    already in HBM; CUDA events on the context stream around the timed
    steps.  Returns a dict (and the open context when keep_open)."""
    import torch
    from croma_fp_b200 import config, native
    fp = native.TracerFP(cfg, path=path)
    crp1, cre1 = seed_rows(fp, cfg)
    fp.set_state_broadcast(nt, crp1, cre1, 1.0e7)
    if dsa:
        fp.set_dsa(config.DsaParams())
    eps = {}
    if emission:
        fp.emission_setup(**native.EMISSION_CONFIG4)
        for k, n in (("syn", "nfreq"), ("ic", "nbins_ic"), ("gamma", "nbins_gamma"), ("nu", "nbins_nu")):
            eps[k] = torch.empty((nt, native.EMISSION_CONFIG4[n]), dtype=torch.float64, device="cuda")
    stream = torch.cuda.ExternalStream(fp.stream())
    emis_events = []

    def step(k, timed):
        isnap = snaps[k]
        launches, ninj = 0, 0
        if dsa:
            sh = {"on_device": 1, "has_dsa": 0}
            for i, key in enumerate(SHOCK_KEYS):
                sh[key] = sh_dev[k, i].data_ptr()
            ninj = fp.dsa_inject(sh, 1.0, float(w.dt[isnap]), "tracer_state")
            launches += fp.last_launch_count()
        if emission:
            if timed:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            fp.emission_run_device(bg_dev[k].data_ptr(), float(w.z[isnap]),
                                   **{kk: t.data_ptr() for kk, t in eps.items()})
            if timed:
                e1.record(stream)
                emis_events.append((e0, e1))
            # 3 GEMMs, the IC table and its weights (z changes every snapshot),
            # the synchrotron plane keys, the radix sort's 4 kernels, the synchrotron
            launches += 12
        fp.snapshot(bg_dev[k].data_ptr(), bg_dev[k + 1].data_ptr(), float(w.z[isnap]), float(w.z[isnap + 1]),
                    True, float(w.dt[isnap]), float(w.elapsed[isnap]), sync=False)
        launches += fp.last_launch_count()
        return launches, ninj

    for k in range(warmup):
        step(k, False)
    fp.sync()
    if kernel_timing:
        fp.set_kernel_timing(True)
        fp.reset_kernel_stats()
    torch.cuda.synchronize()
    clocks = ClockSampler(clock_dev) if clock_dev is not None else None
    if clocks:
        clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches, ninj = 0, []
    ev0.record(stream)
    for k in range(warmup, warmup + steps):
        l, n = step(k, True)
        launches += l
        ninj.append(n)
    ev1.record(stream)
    ev1.synchronize()
    fp.sync()
    torch.cuda.synchronize()
    if clocks:
        clocks.stop()
    out = {"ms": ev0.elapsed_time(ev1), "launches": launches, "dsa_injected_per_step": float(np.mean(ninj)),
           "emission_ms": sum(a.elapsed_time(b) for a, b in emis_events),
           "clocks": clocks.summary() if clocks else None}
    if kernel_timing:
        for kind in ("evolve", "coeff", "secondary"):
            out[kind] = fp.kernel_stats(kind)
        fp.set_kernel_timing(False)
    sched = fp.schedule()
    out["nsub"] = {"min": int(sched["nsub"].min()), "mean": float(sched["nsub"].mean()),
                   "max": int(sched["nsub"].max())}
    out["nbuckets"] = sched["nbuckets"]
    out["sched"] = sched
    if keep_open:
        return out, fp, eps
    fp.close()
    return out


# ---------------------------------------------------------------- e2e through host memory
# share of the host memory left that the e2e measurement's page-locked
# buffers may take (all local ranks together)
E2E_HOST_SHARE = 0.6


def host_bytes_available():
    """Bytes the host can still give this job: MemAvailable of /proc/meminfo,
    capped by the memory cgroup's limit less its usage where one is set
    (cgroup v2, else v1); None when neither can be read."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
                    break
    except (OSError, ValueError, IndexError):
        pass
    for lim_f, use_f in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                         ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            with open(lim_f) as f:
                lim = f.read().strip()
            if lim == "max":
                break
            with open(use_f) as f:
                left = int(lim) - int(f.read().strip())
            avail = left if avail is None else min(avail, left)
            break
        except (OSError, ValueError):
            continue
    return avail


def e2e_tracers(cfg, nt, steps, local_ranks, avail):
    """Tracers of the e2e measurement: all nt, unless the page-locked host
    buffers of the local ranks (spectra and emissivities out, backgrounds and
    shock fields in) would take more than E2E_HOST_SHARE of the host memory
    left (avail bytes); then the largest multiple of 4,096 that fits."""
    from croma_fp_b200 import native
    e = native.EMISSION_CONFIG4
    per_tracer = 8 * (2 * cfg.nb + e["nfreq"] + e["nbins_ic"] + e["nbins_gamma"] + e["nbins_nu"]
                      + 8 * (steps + 2) + len(SHOCK_KEYS) * (steps + 1))
    if avail is None:
        return nt
    fit = int(E2E_HOST_SHARE * avail / max(1, local_ranks) / per_tracer)
    return nt if fit >= nt else max(4096, fit // 4096 * 4096)


def run_e2e(fp, cfg, nt, w, bgs, shocks, snaps, steps):
    """croma_b200_step_host on page-locked host buffers: per step the
    backgrounds and shock fields go up, the emissivities and the evolved
    spectra come back.  Wall time of each (synchronous) call."""
    from croma_fp_b200 import native
    pins = []

    def pinned(shape):
        p = native.PinnedArray(shape, cfg.nb)
        pins.append(p)
        return p.a

    try:
        t0 = time.perf_counter()
        outs = {"crp": pinned((nt, cfg.nb)), "cre": pinned((nt, cfg.nb))}
        for k, n in (("syn", "nfreq"), ("ic", "nbins_ic"), ("gamma", "nbins_gamma"), ("nu", "nbins_nu")):
            outs[k] = pinned((nt, native.EMISSION_CONFIG4[n]))
        nin = steps + 1
        bg_h = [pinned((8, nt)) for _ in range(nin + 1)]
        for k in range(nin + 1):
            bg_h[k][:] = bgs[k]
        sh_h = []
        for k in range(nin):
            arr = pinned((len(SHOCK_KEYS), nt))
            for i, key in enumerate(SHOCK_KEYS):
                arr[i] = shocks[k][key]
            sh_h.append({key: arr[i] for i, key in enumerate(SHOCK_KEYS)} | {"has_dsa": 0})
        t_pin = time.perf_counter() - t0

        def call(k):
            isnap = snaps[k]
            fp.step_host(bg_h[k], bg_h[k + 1], float(w.z[isnap]), float(w.z[isnap + 1]), True, float(w.dt[isnap]),
                         float(w.elapsed[isnap]), shocks=sh_h[k], dsa_mode="tracer_state", outputs=outs)

        call(0)   # untimed: the copy streams and events are created on first use
        times = []
        for k in range(1, nin):
            t0 = time.perf_counter()
            call(k)
            times.append(time.perf_counter() - t0)
        h2d = bg_h[0].nbytes * 2 + sh_h[0]["mach"].nbytes * len(SHOCK_KEYS)
        d2h = sum(a.nbytes for a in outs.values())
        return {"times": times, "h2d": h2d, "d2h": d2h, "pin_s": t_pin}
    finally:
        for p in pins:
            p.free()


# ---------------------------------------------------------------- accuracy and CPU baseline
def accuracy_and_cpu(cfg, w, bgs, shocks, snaps, ntr, nsnap, paths=("fused", "fp32r"), threads=0):
    """The first ntr tracers of the workload through nsnap consecutive steps
    (DSA tracer_state + snapshot) on the reference's own CPU code (oracle/_ref,
    all host threads; the restatement where the reference was not built) and
    on the GPU (each path in `paths`, same inputs, in lockstep): per
    snapshot the max and median relative error over bins above 1e-12 of each
    tracer's peak, the largest particle-number drift and the nsub mismatches;
    emission of the first snapshot (fused path: IC with the reference's own
    table, gamma / neutrino integrals of the reference on the device-built
    kernel tables).  The reference's time per step is the CPU baseline."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from croma_fp_b200 import config, native, synth
    kind = "reference" if pyoracle.reference_available(cfg.nb) else "port"
    ref = pyoracle.ReferenceCPU(cfg, threads=threads) if kind == "reference" else pyoracle.Oracle(cfg)
    cores = ref.threads() if kind == "reference" else 1
    gp, ge = ref.grid(0), ref.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), ntr, cfg.species)
    qpi, qepri = np.zeros_like(crp), np.zeros_like(cre)
    dis = np.zeros(ntr, np.uint8)
    mass = np.full(ntr, 1.0e7)
    fps = {}
    for p in paths:
        fp = native.TracerFP(cfg, path=p)
        crp1, cre1 = seed_rows(fp, cfg)
        fp.set_state_broadcast(ntr, crp1, cre1, 1.0e7)
        fp.set_dsa(config.DsaParams())
        fps[p] = fp
    fps[paths[0]].emission_setup(**native.EMISSION_CONFIG4)
    per_snap = {p: [] for p in paths}
    t_ref, emis = 0.0, None
    try:
        for k in range(nsnap):
            isnap = snaps[k]
            bgc, bgn = bgs[k][:, :ntr].copy(), bgs[k + 1][:, :ntr].copy()
            sh = {key: shocks[k][key][:ntr].copy() for key in SHOCK_KEYS} | {"has_dsa": 0}
            t0 = time.perf_counter()
            ref.dsa_inject(config.DsaParams(), sh, mass, 1.0, float(w.dt[isnap]), 1, 0, crp, cre, qpi, qepri, dis)
            t_dsa = time.perf_counter() - t0
            for fp in fps.values():
                fp.dsa_inject(sh, 1.0, float(w.dt[isnap]), "tracer_state")
            if k == 0:
                emis = emission_check(ref, fps[paths[0]], cfg, bgc, cre, crp, float(w.z[isnap]), kind)
            t0 = time.perf_counter()
            nsub, _, _, _ = ref.snapshot(bgc, bgn, float(w.z[isnap]), float(w.z[isnap + 1]), True, float(w.dt[isnap]),
                                         float(w.elapsed[isnap]), qpi, qepri, crp, cre, mass=mass, dis=dis)
            t_ref += t_dsa + time.perf_counter() - t0
            for p, fp in fps.items():
                fp.snapshot(bgc, bgn, float(w.z[isnap]), float(w.z[isnap + 1]), True, float(w.dt[isnap]),
                            float(w.elapsed[isnap]), sync=True)
                g_crp, g_cre = fp.get_state()
                per_snap[p].append(compare_spectra(g_crp, g_cre, crp, cre, gp[1], ge[1], fp.schedule()["nsub"], nsub))
    finally:
        for fp in fps.values():
            fp.close()
    acc = {"vs": f"reference CPU ({kind}) on the first {ntr} tracers, {nsnap} consecutive snapshots "
                 f"(DSA tracer_state + snapshot)", "tracers": ntr, "snapshots": nsnap, "bar": 1e-6,
           "emission_first_snapshot": emis}
    for p, ps in per_snap.items():
        acc[p] = {"max_rel_err": max(x["max_rel_err"] for x in ps),
                  "median_rel_err": float(np.median([x["median_rel_err"] for x in ps])),
                  "max_particle_number_drift": max(x["drift"] for x in ps),
                  "nsub_mismatches": int(sum(x["nsub_mismatches"] for x in ps)),
                  "per_snapshot_max_rel_err": [x["max_rel_err"] for x in ps]}
    cpu = {"value": ntr * nsnap / t_ref, "unit": UNIT, "cores": cores, "kind": kind,
           "sample": f"{ntr} tracers x {nsnap} consecutive snapshots (DSA tracer_state + IC rows + nsub + "
                     f"buckets + evolve; no emission) in {t_ref:.1f} s"}
    return acc, cpu


def compare_spectra(g_crp, g_cre, crp, cre, dp_p, dp_e, g_nsub, nsub):
    rels, drift = [], 0.0
    for g, r, dp in ((g_crp, crp, dp_p), (g_cre, cre, dp_e)):
        peak = np.max(np.abs(r), axis=1, keepdims=True)
        m = np.abs(r) > 1e-12 * peak
        if m.any():
            rels.append(np.abs(g - r)[m] / np.abs(r)[m])
        ng, nr = g @ dp, r @ dp
        ok = nr != 0
        if ok.any():
            drift = max(drift, float(np.max(np.abs(ng[ok] - nr[ok]) / np.abs(nr[ok]))))
    rel = np.concatenate(rels) if rels else np.zeros(1)
    return {"max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)), "drift": drift,
            "nsub_mismatches": int(np.sum(np.asarray(g_nsub) != np.asarray(nsub)))}


def emission_check(ref, fp, cfg, bg, cre, crp, z, kind):
    """Emission of the post-injection spectra of the first snapshot on the
    GPU against the reference: IC with the reference's own table
    (prepare_ic_kernel_flat + prepare_ic_emission_batch); gamma / neutrino
    with the reference's integrals (prepare_*_emission_cell_major) on the
    device-built kernel tables; synchrotron is pinned by the test suite."""
    from croma_fp_b200 import native, ref_abi
    if kind != "reference":
        return None
    e = native.EMISSION_CONFIG4
    g = fp.emission_run(bg, z, kinds=("ic", "gamma", "nu"))
    out = {}
    _, eps_ic = ref.ic_emission(cre, e["nbins_ic"], z, e["nu_min_ic"], e["nu_max_ic"])
    out["ic_max_rel_err"] = rel_above(g["ic"], eps_ic)
    abi = ref_abi.RefAbi(cfg.nb)
    gp = ref.grid(0)
    for k, fn, lo, hi, nb in (("gamma", "prepare_gamma_kernel_flat_cuda", e["egamma_min"], e["egamma_max"],
                               e["nbins_gamma"]),
                              ("nu", "prepare_neutrino_kernel_flat_cuda", e["enu_min"], e["enu_max"], e["nbins_nu"])):
        table = abi.kernel_table(fn, gp[0], nb, lo, hi)
        r = ref.hadronic_emission(k, crp, bg[0], table, lo, hi)
        out[f"{k}_max_rel_err"] = rel_above(g[k], r)
    out["note"] = "bins above 1e-12 of each tracer's peak; synchrotron pinned by tests/test_emission_tables.py"
    return out


def rel_above(a, b):
    peak = np.max(np.abs(b), axis=1, keepdims=True)
    m = np.abs(b) > 1e-12 * peak
    return float(np.max(np.abs(a - b)[m] / np.abs(b)[m])) if m.any() else 0.0


# ---------------------------------------------------------------- reference arm
def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    load_package()
    from croma_fp_b200 import config, synth
    cfg = workload_config()
    kind = "reference" if pyoracle.reference_available(cfg.nb) else "port"
    ref = pyoracle.ReferenceCPU(cfg) if kind == "reference" else pyoracle.Oracle(cfg)
    cores = ref.threads() if kind == "reference" else 1
    n = args.reference_tracers
    nsteps = args.warmup + args.steps
    snaps = [FIRST_SNAP + k for k in range(nsteps)]
    w, bgs, shocks = make_inputs(cfg, n, snaps, SEED)
    gp, ge = ref.grid(0), ref.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
    qpi, qepri = np.zeros_like(crp), np.zeros_like(cre)
    dis = np.zeros(n, np.uint8)
    mass = np.full(n, 1.0e7)
    times = []
    for k in range(nsteps):
        isnap = snaps[k]
        sh = {key: shocks[k][key] for key in SHOCK_KEYS} | {"has_dsa": 0}
        t0 = time.perf_counter()
        ref.dsa_inject(config.DsaParams(), sh, mass, 1.0, float(w.dt[isnap]), 1, 0, crp, cre, qpi, qepri, dis)
        ref.snapshot(bgs[k], bgs[k + 1], float(w.z[isnap]), float(w.z[isnap + 1]), True, float(w.dt[isnap]),
                     float(w.elapsed[isnap]), qpi, qepri, crp, cre, mass=mass, dis=dis)
        times.append(time.perf_counter() - t0)
    timed = times[args.warmup:] or times
    step_s = float(statistics.median(timed))
    value = n / step_s
    sample = (f"{n} tracers of the workload per step (one snapshot each: DSA tracer_state + IC rows + nsub + "
              f"buckets + evolve on {cores} threads; emission not included), median of {len(timed)} timed steps")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_desc(NTRACER), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def coeff_segments(cfg, nsub):
    """Coefficient segments of a tracer (largest power of two within the
    segment cap and nsub / min_steps), as the schedule kernel derives them."""
    if nsub <= 1 or cfg.coeff_interp_min_steps <= 0:
        return 1
    max_allowed = nsub // cfg.coeff_interp_min_steps
    if max_allowed < 1:
        return 1
    seg = 1
    while seg * 2 <= max(1, cfg.coeff_interp_max_segments) and seg * 2 <= max_allowed:
        seg *= 2
    return min(seg, nsub)


def roofline_fused(cfg, nt, res, steps, fp64_peak, peaks, peak_kind):
    """The steps kernel (dominant) against the live FP64 FMA peak, with its
    HBM view, and the factor / secondary kernels beside it."""
    nb = cfg.nb
    sched = res["sched"]
    nsub = sched["nsub"].astype(np.float64)
    nseg = np.array([coeff_segments(cfg, int(x)) for x in sched["nsub"]], dtype=np.float64)
    ev_ms, ev_n = res["evolve"]
    co_ms, co_n = res["coeff"]
    se_ms, se_n = res["secondary"]
    flops_per_snapshot = float(np.sum(nsub)) * 2 * nb * 11.0
    per_launch = flops_per_snapshot * steps / max(1, ev_n)
    avg_ms = ev_ms / max(1, ev_n)
    achieved = per_launch / (avg_ms / 1e3) / 1e12
    # launch bytes: factored rows (3 nb doubles per segment), N in and out,
    # segment-start proton spectra (the proton launches)
    launches_per_snapshot = max(1, ev_n // steps)
    alg_bytes_snapshot = (float(np.sum(nseg)) * 3 * nb * 8 * 2 + nt * nb * 16 * 2 + float(np.sum(nseg)) * nb * 8)
    alg_bytes_launch = alg_bytes_snapshot / launches_per_snapshot
    # tracer-launches per snapshot: both species over every chunk
    traffic = NCU_DRAM_BYTES_PER_TRACER["steps"] * 2 * nt / launches_per_snapshot if cfg.nb == 512 else None
    ms_total = res["ms"]
    return {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": achieved / fp64_peak, "traffic": traffic,
            "traffic_source": "ncu DRAM bytes per tracer-launch (profiles/steps_kernel_*_full_pipeline_e_p_512.txt) "
                              "x tracers per launch",
            "peak_source": "measured live: croma_b200_fp64_peak (FMA chains on every SM)",
            "kernel": "steps_kernel (proton and electron launches per workspace chunk)",
            "launches": ev_n, "kernel_ms_total": ev_ms, "share_of_step": ev_ms / ms_total,
            "alg_flops_per_launch": per_launch,
            "alg_flops_rule": "per tracer-snapshot: nsub x 2 species x nb x 11 (reference Thomas step)",
            "hbm_view": {"alg_bytes_per_launch": alg_bytes_launch,
                         "achieved_gbs": alg_bytes_launch / (avg_ms / 1e3) / 1e9,
                         "peak_gbs": float(peaks.get("hbm_gbs", 6650.0)), "peak_source": peak_kind},
            "other_kernels": {
                "factor_kernel": {"ms_total": co_ms, "launches": co_n, "share_of_step": co_ms / ms_total},
                "secondary_kernel": {"ms_total": se_ms, "launches": se_n, "share_of_step": se_ms / ms_total},
                "emission": {"ms_total": res["emission_ms"], "share_of_step": res["emission_ms"] / ms_total}}}


def roofline_plain(cfg, nt, res, steps, peaks, peak_kind):
    """The per-step kernel against the HBM copy peak, contract bytes."""
    nb = cfg.nb
    nsub = res["sched"]["nsub"].astype(np.float64)
    ev_ms, ev_n = res["evolve"]
    doubles = (5 + 1) + 5   # electrons: a, b, c, N, source read, N written; protons: no source
    per_launch = float(np.sum(nsub)) * nb * doubles * 8 * steps / max(1, ev_n)
    avg_ms = ev_ms / max(1, ev_n)
    achieved = per_launch / (avg_ms / 1e3) / 1e9
    peak = float(peaks.get("hbm_gbs", 6650.0))
    # tracer-launches per snapshot: both species over every segment slot and chunk
    nslot = 16
    traffic = (NCU_DRAM_BYTES_PER_TRACER["plain_steps"] * 2 * nslot * nt * steps / max(1, ev_n)
               if cfg.nb == 512 else None)
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_kind,
            "traffic_source": "ncu DRAM bytes per tracer-launch (profiles/plain_steps_kernel_electrons_full_pipeline_"
                              "e_p_512.txt) x tracers per launch",
            "frac_meaning": "contract bytes (the reference's per-step data contract) per second; each warp runs "
                            "its slot's sub-steps back to back, so the per-step re-reads hit L2 and DRAM itself "
                            "sees a few per cent of these bytes (traffic)",
            "kernel": "plain_steps_kernel", "launches": ev_n, "kernel_ms_total": ev_ms,
            "share_of_step": ev_ms / res["ms"], "alg_bytes_per_launch": per_launch,
            "alg_bytes_rule": "per tracer-snapshot: nsub x nb x (6 doubles electrons with their secondary "
                              "source + 5 protons without a source)"}


def run_gpu_arm(args):
    import torch
    load_package()
    from croma_fp_b200 import native

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def rank_max(x):
        """The largest x over the ranks (x itself on one GPU)."""
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    cfg = workload_config()
    nt = args.tracers
    nsteps = args.warmup + args.steps
    snaps = [FIRST_SNAP + k for k in range(nsteps)]
    t_in = time.perf_counter()
    w, bgs, shocks = make_inputs(cfg, nt, snaps, SEED + 7919 * rank)
    bg_dev = torch.empty((len(bgs), 8, nt), dtype=torch.float64, device=f"cuda:{local}")
    for k, b in enumerate(bgs):
        bg_dev[k].copy_(torch.from_numpy(b))
    sh_dev = torch.empty((nsteps, len(SHOCK_KEYS), nt), dtype=torch.float64, device=f"cuda:{local}")
    for k in range(nsteps):
        for i, key in enumerate(SHOCK_KEYS):
            sh_dev[k, i].copy_(torch.from_numpy(np.ascontiguousarray(shocks[k][key])))
    torch.cuda.synchronize()
    t_in = time.perf_counter() - t_in
    if dist:
        dist.barrier()

    # ---- the on-chip FP64 path, inputs resident ----
    res, fp, _eps = run_resident("fused", cfg, nt, w, bg_dev, sh_dev, snaps, args.warmup, args.steps,
                                 emission=not args.no_emission, kernel_timing=True, clock_dev=local, keep_open=True)
    if dist:
        dist.barrier()
    ms_max = rank_max(res["ms"])
    value = world * nt * args.steps / (ms_max / 1e3)

    fp64_peak = native.fp64_peak(cfg.nb)
    tuning = {"protons": fp.tuning(0), "electrons": fp.tuning(1)}

    # ---- e2e through host memory: on the same context, or, where the host
    # memory left cannot hold every rank's page-locked buffers for all
    # tracers, on a context of fewer tracers (the same for every rank) ----
    e2e = None
    if not args.no_e2e:
        from croma_fp_b200 import config
        local_ranks = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
        ne = int(-rank_max(-float(e2e_tracers(cfg, nt, args.e2e_steps, local_ranks, host_bytes_available()))))
        ctx, bgs_e, shocks_e = fp, bgs, shocks
        r, e2e_err = None, None
        try:
            if ne < nt:
                fp.close()
                fp = None
                del _eps
                torch.cuda.empty_cache()
                ctx = native.TracerFP(cfg, path="fused")
                crp1, cre1 = seed_rows(ctx, cfg)
                ctx.set_state_broadcast(ne, crp1, cre1, 1.0e7)
                ctx.set_dsa(config.DsaParams())
                ctx.emission_setup(**native.EMISSION_CONFIG4)
                bgs_e = [np.ascontiguousarray(b[:, :ne]) for b in bgs]
                shocks_e = [{k: (np.ascontiguousarray(v[:ne]) if isinstance(v, np.ndarray) else v)
                             for k, v in sh.items()} for sh in shocks]
            # every rank pins its host buffers; the ranks agree on success
            # before the timing reduction, so that one rank's failure cannot
            # leave the others waiting in a collective
            r = run_e2e(ctx, cfg, ne, w, bgs_e, shocks_e, snaps, args.e2e_steps)
        except (MemoryError, RuntimeError) as ex:
            r, e2e_err = None, f"{type(ex).__name__}: {ex}"
        finally:
            if ctx is not fp:
                ctx.close()
        failed = rank_max(1.0 if r is None else 0.0)
        if failed:
            e2e = {"value": None, "unit": UNIT, "error": e2e_err or "failed on another rank"}
    if not args.no_e2e and e2e is None:
        e2e_s = rank_max(statistics.median(r["times"]))
        e2e = {"value": world * ne / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(r["h2d"]),
               "d2h_bytes_per_step": int(r["d2h"]), "host_buffers": "page-locked (croma_b200_host_alloc)",
               "api": "croma_b200_step_host: backgrounds and shock fields up, emissivities and evolved spectra "
                      "down every step, copies overlapped with the kernels",
               "steps": len(r["times"]), "ms_per_step": e2e_s * 1e3, "tracers_per_gpu": ne}
        if ne < nt:
            e2e["note"] = (f"{ne} of the {nt} tracers per GPU: the host memory left could not hold the "
                           f"page-locked buffers of all of them for the {local_ranks} rank(s) on this host")
    if fp is not None:
        fp.close()
        del _eps
    torch.cuda.empty_cache()

    # ---- the plain per-step path on the same workload ----
    plain = None
    if not args.no_plain:
        pr = run_resident("plain", cfg, nt, w, bg_dev, sh_dev, snaps, args.plain_warmup, args.plain_steps,
                          emission=not args.no_emission, kernel_timing=True)
        pr["ms"] = rank_max(pr["ms"])
        pv = world * nt * args.plain_steps / (pr["ms"] / 1e3)
        peaks, peak_kind = measured_peaks()
        plain = {"value": pv, "ms_per_step": pr["ms"] / args.plain_steps, "steps": args.plain_steps,
                 "warmup": args.plain_warmup, "chosen_over_plain": value / pv,
                 "roofline": roofline_plain(cfg, nt, pr, args.plain_steps, peaks, peak_kind),
                 "note": "same steps, inputs and emission; the evolve runs the reference's per-step data contract"}
    fp32r = None
    if not args.no_fp32r:
        fr = run_resident("fp32r", cfg, nt, w, bg_dev, sh_dev, snaps, 1, args.fp32r_steps,
                          emission=not args.no_emission, kernel_timing=True)
        fr["ms"] = rank_max(fr["ms"])
        fv = world * nt * args.fp32r_steps / (fr["ms"] / 1e3)
        fp32r = {"value": fv, "ms_per_step": fr["ms"] / args.fp32r_steps, "steps": args.fp32r_steps, "warmup": 1,
                 "over_fused_fp64": fv / value, "over_plain": (fv / plain["value"]) if plain else None,
                 "steps_kernel_ms_per_step": fr["evolve"][0] / args.fp32r_steps,
                 "fused_fp64_steps_kernel_ms_per_step": res["evolve"][0] / args.steps,
                 "note": "each sub-step solved in FP32 and refined once with an FP64 residual; factors, CC "
                         "weights, spectra and particle budget FP64; accuracy in accuracy.fp32r"}
    peaks, peak_kind = measured_peaks()
    roofline = roofline_fused(cfg, nt, res, args.steps, fp64_peak, peaks, peak_kind)
    del bg_dev, sh_dev
    torch.cuda.empty_cache()

    acc = cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            acc, cpu = accuracy_and_cpu(cfg, w, bgs, shocks, snaps, args.accuracy_tracers, args.accuracy_snaps)
        except (RuntimeError, ValueError, FileNotFoundError, OSError) as e:
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": f"{type(e).__name__}: {e}"}
    secondary = None
    if rank == 0 and world == 1 and not args.no_secondary:
        secondary = {"config1": run_config1(args), "config2": run_config2(args),
                     "heavy_tail": run_heavy_tail(args), "real_histories": run_real_histories(args)}
    serving = None
    if rank == 0 and world == 1 and args.serving_requests > 0:
        serving = run_serving(args)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": dict(workload_desc(nt), parallelism=f"dp{world} (independent tracer shards)",
                           path="fused (on-chip FP64)"),
            "e2e": e2e, "plain": plain, "fp32r": fp32r, "roofline": roofline, "cpu_baseline": cpu, "accuracy": acc,
            "autotuner": tuning, "clocks": res["clocks"], "gpu_launches": int(res["launches"]),
            "kernel_ms": {"evolve": res["evolve"][0], "coeff": res["coeff"][0], "secondary": res["secondary"][0],
                          "emission": res["emission_ms"]},
            "dsa_injected_per_step": res["dsa_injected_per_step"], "nsub": res["nsub"], "nbuckets": res["nbuckets"],
            "input_setup_s": t_in, "secondary": secondary, "serving": serving}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_heavy_tail(args):
    """Uneven sub-step counts: the config-0 background distributions on an
    electron grid over p/(m_e c) in [10, 1000] (128 bins, electron-only,
    direct t_acc), whose nsub spread from 11 to the cap of 500 with a heavy
    tail (median ~12, 90th percentile ~200-370), against the same tracers on
    the full [0.1, 1e6] grid where every nsub is 500.  Reported: throughput,
    the nsub distribution, and the balance of the uneven run: the steps and
    factor kernels' time predicted from the uniform run's cost per tracer
    sub-step and per factored segment, divided by the time measured (1.0:
    the uneven work costs exactly its share, no idle tail)."""
    import torch
    from croma_fp_b200 import config, synth
    nt = args.heavy_tail_tracers
    out = {}
    for name, cfg in (("uniform", config.config0(nsub_max=500)),
                      ("heavy_tail", config.config0(pemin=1.0, pemax=3.0, nsub_max=500))):
        w = synth.Workload(cfg, nt, NSNAP_TIMELINE, seed=SEED + 17)
        snaps = [45 + k for k in range(6)]
        bg = torch.stack([torch.from_numpy(w.background(s_)) for s_ in range(snaps[0], snaps[-1] + 2)]).cuda()
        r = run_resident("fused", cfg, nt, w, bg, None, snaps, 2, 4, emission=False, dsa=False, kernel_timing=True)
        nsub = r["sched"]["nsub"].astype(np.float64)
        nseg = np.array([coeff_segments(cfg, int(x)) for x in r["sched"]["nsub"]], dtype=np.float64)
        out[name] = {"value": nt * 4 / (r["ms"] / 1e3), "ms_per_step": r["ms"] / 4,
                     "nsub_percentiles_0_10_50_90_99_100": [float(x) for x in
                                                            np.percentile(nsub, [0, 10, 50, 90, 99, 100])],
                     "steps_ms_per_step": r["evolve"][0] / 4, "factor_ms_per_step": r["coeff"][0] / 4,
                     "sum_nsub": float(nsub.sum()), "sum_nseg": float(nseg.sum())}
        del bg
    u, h = out["uniform"], out["heavy_tail"]
    c_step = u["steps_ms_per_step"] / u["sum_nsub"]
    c_fac = u["factor_ms_per_step"] / u["sum_nseg"]
    predicted = c_step * h["sum_nsub"] + c_fac * h["sum_nseg"]
    measured = h["steps_ms_per_step"] + h["factor_ms_per_step"]
    out["balance"] = predicted / measured
    out["balance_rule"] = ("(uniform run's steps ms per tracer sub-step x heavy-tail sum nsub + its factor ms per "
                           "segment x heavy-tail sum nseg) / heavy-tail steps + factor ms")
    out["workload"] = (f"{nt} tracers, electron-only, 128 bins, direct t_acc 0.3 Gyr; heavy_tail: electron grid "
                       f"[10, 1e3], uniform: [0.1, 1e6]; 4 timed snapshots after 2")
    return out


# the serving workload's background pool and seed species (name, species mask)
SERVE_POOL_TRACERS = 65536
SERVE_POOL_SNAPS = 201
SERVE_SEEDS = (("electron_only", 2), ("proton_only", 3), ("electron_proton", 3))


def serving_workload(nrequests=48, load=0.7, budget_gb=120.0, max_concurrent=4, seed=20261203,
                     rate_tracer_snaps_per_s=1.7e6, pool_tracers=SERVE_POOL_TRACERS, max_chunk=65536,
                     path="fused"):
    """Config 3, one evolve path: Poisson arrivals of independent tracer runs
    on one GPU.  Each request advances a chunk of tracers through a number of
    snapshots: chunk size log-uniform in [64, 65536], 20..200 snapshots, seed
    species uniform over electron-only / proton-only / electron+proton, 256
    bins, ASA, nsub <= 500; arrivals are Poisson at a rate chosen for a target
    offered load of the device; the server admits requests against a 120 GB
    device-memory budget.  Backgrounds come from one seeded pool shared by all
    requests (each reads a strided window of it); every request starts from
    the seed spectra.  Returns p50 / p99 request latency (submission to
    completion) and the throughput over the whole run."""
    load_package()
    from croma_fp_b200 import config, serve, synth
    rng = np.random.default_rng(seed)
    cfg = config.config1()
    w = synth.Workload(cfg, pool_tracers, SERVE_POOL_SNAPS, seed=seed)
    pool = np.empty((SERVE_POOL_SNAPS, 8, pool_tracers))
    for k in range(SERVE_POOL_SNAPS):
        pool[k] = w.background(k)
    seeds = {}
    from croma_fp_b200 import native
    probe = native.TracerFP(cfg, path="fused")
    gp, ge = probe.grid(0), probe.grid(1)
    probe.close()
    for name, _ in SERVE_SEEDS:
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
        k0 = int(rng.integers(0, SERVE_POOL_SNAPS - ns))
        t_off = int(rng.integers(0, pool_tracers - n + 1))
        name, mask = SERVE_SEEDS[int(kinds[i])]
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


def run_serving(args):
    """Config 3: a Poisson stream of requests through the request server,
    once per evolve path on the same arrival stream; p50 / p99 latency and
    throughput per path."""
    out = {}
    for path in args.serving_paths.split(","):
        out[path] = serving_workload(nrequests=args.serving_requests, path=path)
    return out


def run_real_histories(args):
    """Real tracer histories: the 256 tracers of the reference's tracer_10k
    series in tests/golden/golden_histories.npz (raw snapshot fields read by
    the library's HDF5 reader when the fixture was made), tiled to 65,536
    tracers, backgrounds derived on the device from the raw fields
    (croma_b200_background_prepare), three snapshots from the start of the
    series with the reference's tracer_10k run settings (electron_only, ASA in
    a centred window, eta cap 0.1, no sub-step cap), on-chip FP64 path."""
    import torch
    from croma_fp_b200 import config, native, synth
    fix = np.load(os.path.join(ROOT, "tests", "golden", "golden_histories.npz"))
    prm = json.loads(str(fix["params"]))
    cfg = config.tracer_10k(nb=128)
    reps = 256
    keys = ("temp_K", "density", "bx", "by", "bz", "div_v", "curl_v_prev", "curl_v", "curl_v_next", "l_turb_cm",
            "c_dens", "c_mag", "z_prev", "z_curr", "z_next", "apply_temp_floor", "allow_curl_interp")
    bgs = []
    for k in range(4):
        raw = {}
        for key in keys:
            v = fix[f"s{k}_{key}"]
            raw[key] = np.tile(v, reps) if v.ndim else (int(v) if key.startswith(("apply", "allow")) else float(v))
        bgs.append(native.background_prepare(raw, prm, nb=cfg.nb))
    nt = bgs[0].shape[1]
    mass = np.tile(fix["mass"], reps)
    z, dt = fix["z"], fix["dt"]
    fp = native.TracerFP(cfg, path="fused")
    try:
        gp, ge = fp.grid(0), fp.grid(1)
        crp1, cre1 = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 1, cfg.species)
        fp.set_state(np.repeat(crp1, nt, axis=0), np.repeat(cre1, nt, axis=0), mass=mass)
        bg_dev = [torch.from_numpy(b).cuda() for b in bgs]
        stream = torch.cuda.ExternalStream(fp.stream())
        fp.snapshot(bg_dev[0].data_ptr(), bg_dev[1].data_ptr(), float(z[0]), float(z[1]), True, float(dt[0]),
                    0.0, sync=True)   # warm-up: snapshot 0 -> 1 (and the tuner)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        elapsed = float(dt[0])
        e0.record(stream)
        for k in (1, 2):
            fp.snapshot(bg_dev[k].data_ptr(), bg_dev[k + 1].data_ptr(), float(z[k]), float(z[k + 1]), True,
                        float(dt[k]), elapsed, sync=False)
            elapsed += float(dt[k])
        e1.record(stream)
        e1.synchronize()
        fp.sync()
        ms = e0.elapsed_time(e1)
        nsub = fp.schedule()["nsub"]
    finally:
        fp.close()
    return {"workload": f"{nt} tracers = the fixture's 256 tracer_10k tracers x {reps}, 128 bins, electron_only, "
                        "ASA centred window, eta cap 0.1, snapshots 1 -> 3 of the series (dump0026-0028)",
            "value": nt * 2 / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / 2,
            "nsub_percentiles_0_10_50_90_100": [float(np.percentile(nsub, q)) for q in (0, 10, 50, 90, 100)]}


def run_config2(args):
    """The precision workload (1,048,576 tracers, electron_only, 128 bins,
    TTD, DSA tracer_state on 5 % of tracer-snapshots, the 50-snapshot
    timeline), device-resident: the on-chip FP64, FP32-refined and plain
    paths on the same inputs, and the FP32-refined spectra against the
    on-chip FP64 ones after the same steps (max and median relative error
    over bins above 1e-12 of each tracer's peak, particle-number drift) --
    the FP64 path is held to the reference's own code by the config-2 parity
    test (1,024 tracers x 10 snapshots)."""
    import torch
    from croma_fp_b200 import config, synth
    cfg = config.config2()
    nt, nsnap_timeline = 1 << 20, 50
    snaps = [20 + k for k in range(5)]
    w = synth.Workload(cfg, nt, nsnap_timeline, seed=SEED)
    isn = list(range(snaps[0], snaps[-1] + 2))
    with cf.ThreadPoolExecutor(min(16, os.cpu_count() or 4)) as ex:
        bgs = list(ex.map(w.background, isn))
        shocks = list(ex.map(lambda k: synth.shocks(bgs[k], isn[k], SEED, fraction=DSA_FRACTION),
                             range(len(snaps))))
    bg = torch.stack([torch.from_numpy(b) for b in bgs]).cuda()
    sh = torch.empty((len(snaps), len(SHOCK_KEYS), nt), dtype=torch.float64, device="cuda")
    for k in range(len(snaps)):
        for i, key in enumerate(SHOCK_KEYS):
            sh[k, i].copy_(torch.from_numpy(np.ascontiguousarray(shocks[k][key])))
    rate, states, ms = {}, {}, {}
    for path, warm, steps in (("fused", 1, 4), ("fp32r", 1, 4), ("plain", 1, 2)):
        r, fp, _ = run_resident(path, cfg, nt, w, bg, sh, snaps, warm, steps, emission=False, dsa=True,
                                keep_open=True)
        try:
            if path != "plain":
                states[path] = fp.get_state() + (fp.schedule()["nsub"],)
            dp = (fp.grid(0)[1], fp.grid(1)[1])
        finally:
            fp.close()
        rate[path] = nt * steps / (r["ms"] / 1e3)
        ms[path] = r["ms"] / steps
    del bg, sh
    f, q = states["fused"], states["fp32r"]
    err = compare_spectra(q[0], q[1], f[0], f[1], dp[0], dp[1], q[2], f[2])
    return {"workload": "precision: 1,048,576 tracers, electron_only, 128 bins, TTD, DSA tracer_state on 5 % of "
                        "tracer-snapshots (Mach U[2,5]), snapshots 20.. of the z=1->0 50-snapshot timeline, no "
                        "emission", "fused": rate["fused"], "fp32r": rate["fp32r"], "plain": rate["plain"],
            "chosen_over_plain": rate["fused"] / rate["plain"], "ms_per_step": ms,
            "fp32r_vs_fused_fp64": {"after_steps": 5, "max_rel_err": err["max_rel_err"],
                                    "median_rel_err": err["median_rel_err"],
                                    "max_particle_number_drift": err["drift"],
                                    "nsub_mismatches": err["nsub_mismatches"], "bar": 1e-6},
            "steps": {"fused": 4, "fp32r": 4, "plain": 2}}


def run_config1(args):
    """The batching workload (65,536 tracers, e+p, 256 bins, ASA, no DSA or
    emission): fused and plain, device-resident."""
    import torch
    from croma_fp_b200 import config
    cfg = config.config1()
    nt = 65536
    snaps = [5 + k for k in range(8)]
    from croma_fp_b200 import synth
    w = synth.Workload(cfg, nt, NSNAP_TIMELINE, seed=SEED)
    bg = torch.stack([torch.from_numpy(w.background(s)) for s in range(snaps[0], snaps[-1] + 2)]).cuda()
    f = run_resident("fused", cfg, nt, w, bg, None, snaps, 3, 5, emission=False, dsa=False, kernel_timing=True)
    p = run_resident("plain", cfg, nt, w, bg, None, snaps, 1, 2, emission=False, dsa=False)
    vf, vp = nt * 5 / (f["ms"] / 1e3), nt * 2 / (p["ms"] / 1e3)
    return {"workload": "batching: 65,536 tracers, electron_proton, 256 bins, ASA, nsub <= 500 (no DSA, no "
                        "emission)", "fused": vf, "plain": vp, "chosen_over_plain": vf / vp,
            "fused_kernel_ms_per_step": {k: f[k][0] / 5 for k in ("evolve", "coeff", "secondary")},
            "nsub": f["nsub"], "steps": {"fused": 5, "plain": 2}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tracers", type=int, default=NTRACER)
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--plain-warmup", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--accuracy-tracers", type=int, default=4096)
    ap.add_argument("--accuracy-snaps", type=int, default=5)
    ap.add_argument("--reference-tracers", type=int, default=4096)
    ap.add_argument("--fp32r-steps", type=int, default=3)
    ap.add_argument("--no-fp32r", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-emission", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--heavy-tail-tracers", type=int, default=262144)
    ap.add_argument("--serving-requests", type=int, default=48)
    ap.add_argument("--serving-paths", default="fused", help="comma-separated: fused, fp32r, plain")
    ap.add_argument("--serving-only", action="store_true", help="run only the serving workload, one JSON line")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.serving_only:
        load_package()
        print(json.dumps({"serving": run_serving(args)}), flush=True)
        return 0
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
