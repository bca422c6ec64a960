"""Benchmark: tracer-snapshot updates per second of the Fokker-Planck update.

Workload (one "step" = one snapshot of every tracer on a GPU): 65,536
seeded tracers per GPU, electron + proton spectra with 256 momentum bins
each (protons p/(m_p c) in [1e-2, 1e6], electrons in [1e-1, 1e6]), ASA
reacceleration, hadronic secondary electrons, sub-step cap 500, snapshots
of a 100-snapshot z = 1 -> 0 timeline.  The spectra (2 x 256 x 65,536
doubles = 268 MB) exceed the 126 MB L2, so no flush is needed between
steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--path plain|fused]
    python bench.py --impl reference      # the reference's CPU code, same workload

Prints one JSON line (rank 0).  ``value`` is device-timed throughput with
inputs resident in HBM; ``e2e`` runs the same snapshots through the C ABI
with host buffers (background H2D, spectra up and down every snapshot, as
the reference's rank-state path does).
"""
from __future__ import annotations

import argparse
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
NTRACER = 65536
NSNAP_TIMELINE = 100
SEED = 20261203
METRIC = "tracer-snapshot updates/s at <=1e-6 rel err vs FP64, chosen vs plain; p50/p99 latency"
UNIT = "tracer-snapshot updates/s"
# DRAM bytes (read + write) of one steps_kernel launch per tracer, mean of the
# proton and electron launches of an ncu capture of this workload at 32,768
# tracers (profiles/steps_factor_secondary_batching_e_p_256.txt); traffic
# scales with the tracer count (every tracer moves its own rows).
NCU_DRAM_BYTES_PER_TRACER_STEPS_LAUNCH = (3.347485e9 + 1.122321e9 + 4.431413e9 + 0.077046e9) / 2 / 32768
# plain_steps_kernel DRAM read + write per tracer per launch (one segment slot
# of 31.25 sub-steps), mean of the proton and electron launches, from one ncu
# capture at 32,768 tracers of the same workload
NCU_DRAM_BYTES_PER_TRACER_PLAIN_LAUNCH = (272.135680e6 + 48.561664e6 + 339.285760e6 + 53.114880e6) / 2 / 32768


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
    return config.config1()


def workload_desc(ntracer):
    return {"workload": "batching: electron_proton with pp secondaries, 256 bins/species, ASA Dpp, "
                        "nsub capped at 500, z=1->0 over 100 snapshots",
            "tracers_per_gpu": ntracer, "bins_per_species": 256, "species": "electron_proton",
            "dpp_mode": "asa", "nsub_max": 500, "precision": "fp64",
            "l2_policy": "inputs larger than L2 (268 MB of spectra per GPU)"}


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


# ---------------------------------------------------------------- CPU baseline
def cpu_reference_rate(cfg, budget_s=12.0, max_tracers=NTRACER):
    """Reference CPU code (oracle/_ref, all host threads) on a bounded sample
    of the workload: one snapshot of n tracers, n doubled until the snapshot
    takes >= budget_s / 4.  The per-snapshot IC-cooling rows (independent of
    the tracer count) are timed separately and the rate is extrapolated to
    the full tracer count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    load_package()
    from croma_fp_b200 import synth
    kind = "reference" if pyoracle.reference_available(cfg.nb) else "port"
    impl = pyoracle.ReferenceCPU(cfg) if kind == "reference" else pyoracle.Oracle(cfg)
    cores = os.cpu_count() or 1
    w = synth.Workload(cfg, max_tracers, NSNAP_TIMELINE, seed=SEED)
    isnap = 10
    t0 = time.perf_counter()
    impl.ic_row(float(w.z[isnap]))
    impl.ic_row(float(w.z[isnap + 1]))
    t_ic = time.perf_counter() - t0
    gp, ge = impl.grid(0), impl.grid(1)
    n = 64
    spent = 0.0
    while True:
        bgc = w.background(isnap)[:, :n].copy()
        bgn = w.background(isnap + 1)[:, :n].copy()
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        crp0, cre0 = crp.copy(), cre.copy()
        q = np.zeros_like(crp)
        t0 = time.perf_counter()
        nsub, _, _, _ = impl.snapshot(bgc, bgn, float(w.z[isnap]), float(w.z[isnap + 1]), True,
                                      float(w.dt[isnap]), float(w.elapsed[isnap]), q, np.zeros_like(cre), crp,
                                      cre, mass=w.mass[:n])
        dt = time.perf_counter() - t0
        spent += dt
        if dt >= budget_s / 4 or n >= max_tracers or spent > budget_s:
            break
        n *= 2
    per_tracer = max(dt - t_ic, 1e-9) / n
    t_full = t_ic + per_tracer * max_tracers
    check = {"w": w, "isnap": isnap, "bgc": bgc, "bgn": bgn, "crp0": crp0, "cre0": cre0, "crp": crp,
             "cre": cre, "nsub": nsub, "dp": (gp[1], ge[1]), "kind": kind}
    return {"value": max_tracers / t_full, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"1 snapshot x {n} tracers in {dt:.2f} s (IC rows {t_ic:.2f} s/snapshot), "
                      f"extrapolated to {max_tracers} tracers per snapshot"}, dt, n, check


def accuracy_vs_reference(cfg, path, chk):
    """The GPU path on the CPU baseline's own sample (same tracers, inputs and
    snapshot) against the reference CPU's result: max and median relative
    error per bin (bins above 1e-12 of each tracer's peak), the largest
    particle-number drift |sum N dp - ref| / ref per tracer and species, and
    the nsub mismatches (which must be 0)."""
    load_package()
    from croma_fp_b200 import native
    w, isnap = chk["w"], chk["isnap"]
    n = chk["crp0"].shape[0]
    fp = native.TracerFP(cfg, path=path)
    try:
        fp.set_state(chk["crp0"], chk["cre0"], mass=w.mass[:n])
        fp.snapshot(chk["bgc"], chk["bgn"], float(w.z[isnap]), float(w.z[isnap + 1]), True, float(w.dt[isnap]),
                    float(w.elapsed[isnap]), sync=True)
        g_crp, g_cre = fp.get_state()
        g_nsub = fp.schedule()["nsub"]
    finally:
        fp.close()
    rels, drift = [], 0.0
    for g, r, dp in ((g_crp, chk["crp"], chk["dp"][0]), (g_cre, chk["cre"], chk["dp"][1])):
        peak = np.max(np.abs(r), axis=1, keepdims=True)
        m = np.abs(r) > 1e-12 * peak
        if m.any():
            rels.append((np.abs(g - r)[m] / np.abs(r)[m]))
        ng, nr = g @ dp, r @ dp
        ok = nr != 0
        if ok.any():
            drift = max(drift, float(np.max(np.abs(ng[ok] - nr[ok]) / np.abs(nr[ok]))))
    rel = np.concatenate(rels) if rels else np.zeros(1)
    return {"vs": f"reference CPU ({chk['kind']}) on the CPU baseline's sample", "tracers": n,
            "max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
            "max_particle_number_drift": drift, "nsub_mismatches": int(np.sum(g_nsub != chk["nsub"])),
            "bar": 1e-6}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg = workload_config()
    vals = []
    first = None
    for _ in range(args.warmup + args.steps):
        res, dt, n, _ = cpu_reference_rate(cfg, budget_s=max(2.0, 60.0 / max(1, args.steps + args.warmup)))
        vals.append(res["value"])
        first = first or res
    timed = vals[args.warmup:] or vals
    value = float(statistics.median(timed))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": NTRACER / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_desc(NTRACER), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": first["cores"], "kind": first["kind"],
                             "sample": first["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def coeff_segments(cfg, nsub, allow=True):
    """Coefficient segments of a tracer (largest power of two within the
    segment cap and nsub / min_steps), as the schedule kernel derives them."""
    if not allow or nsub <= 1 or cfg.coeff_interp_min_steps <= 0:
        return 1
    max_seg = max(1, cfg.coeff_interp_max_segments)
    max_allowed = nsub // cfg.coeff_interp_min_steps
    if max_allowed < 1:
        return 1
    seg = 1
    while seg * 2 <= max_seg and seg * 2 <= max_allowed:
        seg *= 2
    return min(seg, nsub)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return json.load(open(p)), "measured"
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def run_gpu_arm(args):
    import torch
    load_package()
    from croma_fp_b200 import native, synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    cfg = workload_config()
    nt = args.tracers
    w = synth.Workload(cfg, nt, NSNAP_TIMELINE, seed=SEED + 7919 * rank)
    fp = native.TracerFP(cfg, path=args.path, device=local)
    gp, ge = fp.grid(0), fp.grid(1)
    crp0, cre0 = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    fp.set_state(crp0, cre0, mass=w.mass)

    nsteps_total = args.warmup + args.steps
    first = 5
    snaps = list(range(first, first + nsteps_total))
    bg_dev = torch.empty((nsteps_total + 1, 8, nt), dtype=torch.float64, device=f"cuda:{local}")
    for k in range(nsteps_total + 1):
        bg_dev[k].copy_(torch.from_numpy(w.background(first + k)))
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(fp.stream(), device=f"cuda:{local}")

    def do_snapshot(k, isnap):
        fp.snapshot(bg_dev[k].data_ptr(), bg_dev[k + 1].data_ptr(), float(w.z[isnap]),
                    float(w.z[isnap + 1]), True, float(w.dt[isnap]), float(w.elapsed[isnap]), sync=False)
        return fp.last_launch_count()

    for k in range(args.warmup):
        do_snapshot(k, snaps[k])
    fp.sync()
    fp.set_kernel_timing(True)
    fp.reset_kernel_stats()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches = 0
    ev0.record(stream)
    for k in range(args.warmup, nsteps_total):
        launches += do_snapshot(k, snaps[k])
    ev1.record(stream)
    ev1.synchronize()
    fp.sync()
    torch.cuda.synchronize()
    clocks.stop()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    evolve_ms, evolve_n = fp.kernel_stats("evolve")
    coeff_ms, coeff_n = fp.kernel_stats("coeff")
    sec_ms, sec_n = fp.kernel_stats("secondary")
    fp.set_kernel_timing(False)
    sched = fp.schedule()
    ms_max = ms
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * nt * args.steps / (ms_max / 1e3)

    # ---- e2e through the C ABI with page-locked host buffers ----
    def pinned(shape):
        return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    crp_h, cre_h = pinned((nt, cfg.nb)), pinned((nt, cfg.nb))
    fp.get_state(crp_h, cre_h)
    mass_h = pinned((nt,))
    mass_h[:] = w.mass
    bg_host = []
    for k in range(min(args.steps, 3) + 1):
        b = pinned((8, nt))
        b[:] = w.background(first + k)
        bg_host.append(b)
    # (a) the pipelined host-buffer call: chunk uploads and downloads on two
    # copy streams overlap the evolve; one untimed call creates its streams
    nsteps_e2e = min(args.steps, 3)
    def host_args(k):
        isnap = snaps[k]
        return (bg_host[k], bg_host[k + 1], float(w.z[isnap]), float(w.z[isnap + 1]), True,
                float(w.dt[isnap]), float(w.elapsed[isnap]))
    fp.snapshot_host(crp_h, cre_h, *host_args(0), mass=mass_h)
    e2e_times = []
    for k in range(nsteps_e2e):
        t0 = time.perf_counter()
        fp.snapshot_host(crp_h, cre_h, *host_args(k), mass=mass_h)
        e2e_times.append(time.perf_counter() - t0)
    h2d = crp_h.nbytes + cre_h.nbytes + mass_h.nbytes + bg_host[0].nbytes * 2
    d2h = crp_h.nbytes + cre_h.nbytes
    # (b) the same through set_state / snapshot / get_state in turn
    seq_times = []
    for k in range(nsteps_e2e):
        t0 = time.perf_counter()
        fp.set_state(crp_h, cre_h, mass=mass_h)
        fp.snapshot(*host_args(k), sync=False)
        fp.get_state(crp_h, cre_h)
        seq_times.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e_times)
    seq_s = statistics.median(seq_times)
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
        t = torch.tensor([seq_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        seq_s = float(t.item())
    e2e_value = world * nt / e2e_s

    # ---- roofline of the dominant kernel ----
    peaks, peak_kind = measured_peaks()
    nsub = sched["nsub"].astype(np.float64)
    nb = cfg.nb
    nspecies = 2
    if args.path == "plain":
        # algorithmic bytes of the sub-step kernels (reference data contract):
        # a, b, c and N read, N written per row per sub-step, plus the source
        # of a species that has one (electrons: the secondaries; protons: none
        # in this workload)
        e_src = 1 if cfg.species == "electron_proton" else 0
        doubles = (5 + e_src) + 5
        bytes_per_snapshot = float(np.sum(nsub)) * nb * doubles * 8
        alg_bytes_total = bytes_per_snapshot * args.steps
        per_launch = alg_bytes_total / max(1, evolve_n)
        avg_launch_ms = evolve_ms / max(1, evolve_n)
        achieved = per_launch / (avg_launch_ms / 1e3) / 1e9
        peak = float(peaks.get("hbm_gbs", 6650.0))
        traffic = NCU_DRAM_BYTES_PER_TRACER_PLAIN_LAUNCH * nt if args.tracers == NTRACER else None
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                    "traffic_note": "each warp runs its slot's sub-steps back to back, so the per-step "
                                    "re-reads of the contract hit L2; DRAM sees ~3 % of the contract bytes",
                    "kernel": "plain_steps_kernel", "launches": evolve_n,
                    "kernel_ms_total": evolve_ms, "share_of_step": evolve_ms / ms if ms > 0 else None,
                    "alg_bytes_per_launch": per_launch,
                    "alg_bytes_rule": "per tracer-snapshot: nsub x nb x (6 doubles electrons with their "
                                      "secondary source + 5 protons without a source)"}
    else:
        # The steps kernel runs every sub-step with the spectrum and the factored
        # rows in registers: the bound is the FP64 pipe.  Algorithmic flops are
        # the reference's Thomas step per row per sub-step (RHS FMA, denominator
        # FMA, back-substitution FMA, 2 divides: 9 flops + 2 divides, counted 11)
        # over both species and every sub-step of the schedule.  Its DRAM traffic
        # is the factored rows of each segment (written by the factor kernel),
        # the spectra and the segment-start proton spectra.
        flops_per_snapshot = float(np.sum(nsub)) * nspecies * nb * 11.0
        per_launch = flops_per_snapshot * args.steps / max(1, evolve_n)
        avg_launch_ms = evolve_ms / max(1, evolve_n)
        achieved = per_launch / (avg_launch_ms / 1e3) / 1e12
        peak = native.fp64_peak(cfg.nb)
        nseg = np.array([coeff_segments(cfg, int(n)) for n in sched["nsub"]], dtype=np.float64)
        # bytes the steps launches must move: factored rows (3 x nb doubles per
        # segment), N in and out, segment-start proton spectra (proton launch)
        alg_bytes_launch = (float(np.sum(nseg)) * (3 * nb * 8) * nspecies + nt * nb * 16 * nspecies
                            + float(np.sum(nseg)) * nb * 8) / nspecies
        traffic = (NCU_DRAM_BYTES_PER_TRACER_STEPS_LAUNCH * nt
                   if NCU_DRAM_BYTES_PER_TRACER_STEPS_LAUNCH and args.tracers == NTRACER else None)
        _, npmin = fp.secondary_kernel()
        sec_flops = float(np.sum(nseg)) * 2.0 * float(np.sum(nb - np.asarray(npmin))) * args.steps
        roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "peak_source": "measured live: croma_b200_fp64_peak (FMA chains on every SM)",
                    "kernel": "steps_kernel (one proton and one electron launch per snapshot)",
                    "launches": evolve_n, "kernel_ms_total": evolve_ms,
                    "share_of_step": evolve_ms / ms if ms > 0 else None,
                    "alg_flops_per_launch": per_launch,
                    "alg_flops_rule": "per tracer-snapshot: nsub x 2 species x nb x 11 (reference Thomas)",
                    "hbm_view": {"alg_bytes_per_launch": alg_bytes_launch,
                                 "achieved_gbs": alg_bytes_launch / (avg_launch_ms / 1e3) / 1e9,
                                 "peak_gbs": float(peaks.get("hbm_gbs", 6650.0)),
                                 "peak_source": peak_kind},
                    "other_kernels": {
                        "factor_kernel": {"ms_total": coeff_ms, "launches": coeff_n,
                                          "share_of_step": coeff_ms / ms if ms > 0 else None},
                        "secondary_kernel": {"ms_total": sec_ms, "launches": sec_n,
                                             "share_of_step": sec_ms / ms if ms > 0 else None,
                                             "achieved_tflops": sec_flops / (sec_ms / 1e3) / 1e12
                                             if sec_ms > 0 else None,
                                             "frac": (sec_flops / (sec_ms / 1e3) / 1e12) / peak
                                             if sec_ms > 0 else None}}}

    serving = None
    if rank == 0 and world == 1 and not args.no_serving:
        # p50 / p99 request latency of the serving workload (Poisson arrivals
        # of tracer chunks), a bounded sample run after the timed region
        fp.close()
        from croma_fp_b200 import serve_bench
        serving = serve_bench.run(nrequests=args.serving_requests)
    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _, _, chk = cpu_reference_rate(cfg, budget_s=args.cpu_budget)
        except Exception as e:  # the checker library may be absent
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable",
                   "sample": f"{type(e).__name__}: {e}"}
        else:
            try:
                accuracy = accuracy_vs_reference(cfg, args.path, chk)
            except (RuntimeError, ValueError) as e:  # native.CromaError is a RuntimeError
                accuracy = {"error": f"{type(e).__name__}: {e}"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": dict(workload_desc(nt), parallelism=f"dp{world} (independent tracer shards)",
                           path=args.path),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "host_buffers": "page-locked",
                    "api": "croma_b200_snapshot_host (copies overlapped with the evolve)",
                    "sequential": {"value": world * nt / seq_s,
                                   "api": "croma_b200_set_state/snapshot/get_state in turn"}},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "accuracy": accuracy,
            "serving": serving,
            "clocks": clocks.summary(),
            "gpu_launches": int(launches),
            "kernel_ms": {"evolve": evolve_ms, "coeff": coeff_ms, "secondary": sec_ms},
            "nsub": {"min": int(nsub.min()), "mean": float(nsub.mean()), "max": int(nsub.max())},
            "nbuckets": sched["nbuckets"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    fp.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="fused", choices=["plain", "fused"])
    ap.add_argument("--tracers", type=int, default=NTRACER)
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=16)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
