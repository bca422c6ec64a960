"""Host-buffer snapshot with overlapped copies (croma_b200_snapshot_host).

The pipelined call must give what set_state + snapshot + get_state give:
the golden fixtures (the reference's own outputs) within the evolve bar, and
bit for bit the result of the three separate calls on a synthetic batch,
whatever the chunking (tracers are independent, so a chunk boundary changes
no arithmetic).  A species the mask does not evolve is not copied back and
its host rows are left as they were.
"""
import numpy as np
import pytest

from conftest import load_package
from golden_io import Case, rel_err

load_package()
from croma_fp_b200 import config, native, synth  # noqa: E402

SPECTRA_RTOL = 1e-10
pytestmark = pytest.mark.gpu


def _pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out, t


@pytest.mark.parametrize("chunks", [0, 3])
@pytest.mark.parametrize("name", ["c0_direct", "c1_asa256", "c1_etacap", "c2_ttd_spect_window"])
def test_snapshot_host_matches_reference(name, chunks):
    c = Case(name)
    d = c.d
    fp = native.TracerFP(c.cfg, path="fused")
    try:
        crp = np.ascontiguousarray(d["crp0"], dtype=np.float64).copy()
        cre = np.ascontiguousarray(d["cre0"], dtype=np.float64).copy()
        for k in range(c.nrun):
            fp.snapshot_host(crp, cre, *c.snapshot_args(k), mass=d["mass"], chunks=chunks)
            sched = fp.schedule()
            assert np.array_equal(sched["nsub"], d[f"nsub_{k}"])
            e = rel_err(cre, d[f"cre_{k}"])
            assert e <= SPECTRA_RTOL, f"electron spectra rel err {e:.3e} at step {k}"
            if np.any(d[f"crp_{k}"]):
                e = rel_err(crp, d[f"crp_{k}"])
                assert e <= SPECTRA_RTOL, f"proton spectra rel err {e:.3e} at step {k}"
    finally:
        fp.close()


def _batch(cfg, n, seed):
    w = synth.Workload(cfg, n, 100, seed=seed)
    probe = native.TracerFP(cfg, path="fused")
    gp, ge = probe.grid(0), probe.grid(1)
    probe.close()
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
    return w, crp, cre


@pytest.mark.parametrize("chunks", [0, 5])
def test_snapshot_host_bitwise_equals_separate_calls(chunks):
    cfg = config.config1(nb=256)
    n = 9000          # >= 8192: the default split is 1125 / 6750 / 1125
    w, crp0, cre0 = _batch(cfg, n, 77)
    args = []
    for k in range(2):
        i = 40 + k
        args.append((w.background(i), w.background(i + 1), float(w.z[i]), float(w.z[i + 1]), True,
                     float(w.dt[i]), float(w.elapsed[i])))
    ref = native.TracerFP(cfg, path="fused")
    ref.set_state(crp0, cre0, mass=w.mass)
    for a in args:
        ref.snapshot(*a, sync=True)
    r_crp, r_cre = ref.get_state()
    ref.close()

    fp = native.TracerFP(cfg, path="fused")
    try:
        crp, keep_p = _pinned(crp0)
        cre, keep_e = _pinned(cre0)
        for a in args:
            fp.snapshot_host(crp, cre, *a, mass=w.mass, chunks=chunks)
        assert np.array_equal(crp, r_crp)
        assert np.array_equal(cre, r_cre)
        # the resident state is the evolved state too
        g_crp, g_cre = fp.get_state()
        assert np.array_equal(g_crp, r_crp) and np.array_equal(g_cre, r_cre)
    finally:
        fp.close()
    del keep_p, keep_e


def test_snapshot_host_electron_only_leaves_proton_rows():
    cfg = config.config1(nb=128, species="electron_only")
    n = 600
    w, crp0, cre0 = _batch(cfg, n, 78)
    i = 25
    a = (w.background(i), w.background(i + 1), float(w.z[i]), float(w.z[i + 1]), True,
         float(w.dt[i]), float(w.elapsed[i]))
    ref = native.TracerFP(cfg, path="fused")
    ref.set_state(crp0, cre0, mass=w.mass)
    ref.snapshot(*a, sync=True)
    _, r_cre = ref.get_state()
    ref.close()
    fp = native.TracerFP(cfg, path="fused")
    try:
        sentinel = np.full_like(crp0, -7.0)
        crp = sentinel.copy()
        cre = cre0.copy()
        # the proton rows uploaded are the sentinel; they are not evolved
        # (mask 2) and so not copied back over the host rows
        fp.snapshot_host(crp, cre, *a, mass=w.mass, chunks=2)
        assert np.array_equal(cre, r_cre)
        assert np.array_equal(crp, sentinel)
    finally:
        fp.close()
