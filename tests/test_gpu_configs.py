"""Parity on the benchmark configurations themselves, not only on the small
golden fixtures: multi-snapshot runs of each configuration's workload
against the oracle (the CPU restatement, pinned bit for bit to the
reference's own CPU code by tests/test_oracle_pin.py), compared after every
snapshot.

* config 0 (plain FP64 method): 1,024 tracers x the full 100-snapshot
  timeline, electron-only, 128 bins, direct t_acc = 0.3 Gyr; the plain and
  the on-chip path in lockstep with the oracle.
* config 1 (batching): 256 tracers, e+p, 256 bins, ASA, nsub <= 500, 6
  snapshots; all three paths.
* config 2 (precision): TTD, 128 bins, DSA tracer_state injection on 5 % of
  tracer-snapshots (Mach U[2, 5]) before each of 10 snapshots of the
  configuration's 50-snapshot timeline; FP64 paths at 1e-10, the
  FP32-refined path at 1e-6.
* config 4 (full pipeline): 64 tracers, e+p with secondaries, 512 bins, ASA,
  DSA on 10 % of tracer-snapshots, 3 snapshots; all three paths.

Bars: nsub / n_on / bucket ids bit-exact on every snapshot; spectra within
1e-10 relative (FP64 paths) or 1e-6 (FP32-refined) on bins above 1e-12 of
each tracer's peak; the particle number sum N dp within the same bar.
"""
import numpy as np
import pytest

from conftest import load_package
from golden_io import rel_err

load_package()
from croma_fp_b200 import config, native, synth  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = {"plain": 1e-10, "fused": 1e-10, "fp32r": 1e-6}


def _oracle(cfg):
    import pyoracle
    return pyoracle.Oracle(cfg)


def _drift(g, r, dp):
    ng, nr = g @ dp, r @ dp
    ok = nr != 0
    return float(np.max(np.abs(ng[ok] - nr[ok]) / np.abs(nr[ok]))) if ok.any() else 0.0


def _lockstep(cfg, nt, first, nsnap, seed, paths, dsa_fraction=0.0, timeline=100):
    """Runs the oracle and one GPU context per path side by side over
    snapshots [first, first + nsnap) of a timeline-snapshot z = 1 -> 0
    timeline; returns the worst spectral error per path."""
    o = _oracle(cfg)
    w = synth.Workload(cfg, nt, timeline, seed=seed)
    gp, ge = o.grid(0), o.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    qpi, qepri = np.zeros_like(crp), np.zeros_like(cre)
    dis = np.zeros(nt, np.uint8)
    prm = config.DsaParams()
    ctx = {}
    for p in paths:
        fp = native.TracerFP(cfg, path=p)
        fp.set_state(crp, cre, mass=w.mass)
        if dsa_fraction > 0.0:
            fp.set_dsa(prm)
        ctx[p] = fp
    worst = {p: 0.0 for p in paths}
    injected = 0
    try:
        for k in range(nsnap):
            isnap = first + k
            args = w.snapshot_args(isnap)
            if dsa_fraction > 0.0:
                sh = synth.shocks(args[0], isnap, seed, fraction=dsa_fraction)
                n_or = o.dsa_inject(prm, sh, w.mass, 1.0, args[5], 1, 0, crp, cre, qpi, qepri, dis)
                injected += n_or
                for p, fp in ctx.items():
                    assert fp.dsa_inject(sh, 1.0, args[5], "tracer_state") == n_or, f"{p} injection count"
            nsub, non, bid, _ = o.snapshot(*args, qpi, qepri, crp, cre, mass=w.mass, dis=dis)
            for p, fp in ctx.items():
                fp.snapshot(*args, sync=True)
                sched = fp.schedule()
                tag = f"{p} snapshot {isnap}"
                assert np.array_equal(sched["nsub"], nsub), tag
                assert np.array_equal(sched["non"], non), tag
                assert np.array_equal(sched["bucket_ids"], bid), tag
                g_crp, g_cre = fp.get_state()
                e = rel_err(g_cre, cre)
                assert _drift(g_cre, cre, ge[1]) <= RTOL[p], tag
                if np.any(crp):
                    e = max(e, rel_err(g_crp, crp))
                    assert _drift(g_crp, crp, gp[1]) <= RTOL[p], tag
                assert e <= RTOL[p], f"{tag}: spectra rel err {e:.3e}"
                worst[p] = max(worst[p], e)
    finally:
        for fp in ctx.values():
            fp.close()
    if dsa_fraction > 0.0:
        assert injected > 0
    return worst


def test_config0_full_timeline_1024_tracers():
    worst = _lockstep(config.config0(nsub_max=500), 1024, 0, 100, 20261, ["plain", "fused"])
    print("config 0, 1024 tracers x 100 snapshots, worst rel err:", worst)


def test_config1_batching_256_tracers_6_snapshots():
    worst = _lockstep(config.config1(), 256, 5, 6, 20263, ["plain", "fused", "fp32r"])
    print("config 1, 256 tracers x 6 snapshots, worst rel err:", worst)


def test_config2_ttd_with_dsa_10_snapshots():
    worst = _lockstep(config.config2(), 1024, 20, 10, 20262, ["plain", "fused", "fp32r"], dsa_fraction=0.05,
                      timeline=50)
    print("config 2, 1024 tracers x 10 snapshots of the 50-snapshot timeline with DSA, worst rel err:", worst)


def test_config4_full_pipeline_64_tracers():
    worst = _lockstep(config.config4(), 64, 30, 3, 20264, ["plain", "fused", "fp32r"], dsa_fraction=0.1)
    print("config 4, 64 tracers x 3 snapshots with DSA, worst rel err:", worst)
