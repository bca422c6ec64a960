"""Edge cases of the evolve paths on the GPU.

* One tracer (a fraction of a warp group and of a block) against the oracle.
* A workspace too small for the batch: the tracers run in chunks of 5 (37
  tracers: chunks that do not divide the batch), bit for bit equal to the
  unchunked run, on both paths and with the eta cap (one segment per launch).
* Spectra that are zero stay exactly zero (no NaN from the implicit solve).
* Invalid calls fail with an error code and a message, and leave the context
  usable.
"""
import dataclasses

import numpy as np
import pytest

from conftest import load_package
from golden_io import rel_err

load_package()
from croma_fp_b200 import config, native, synth  # noqa: E402

pytestmark = pytest.mark.gpu


def _inputs(cfg, n, seed):
    w = synth.Workload(cfg, n, 100, seed=seed)
    import pyoracle
    o = pyoracle.Oracle(cfg)
    gp, ge = o.grid(0), o.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
    return w, o, crp, cre


def _run(cfg, path, w, crp, cre, snaps, limit=None):
    fp = native.TracerFP(cfg, path=path)
    try:
        if limit is not None:
            fp.set_workspace_limit(limit)
        fp.set_state(crp, cre, mass=w.mass)
        for i in snaps:
            fp.snapshot(*w.snapshot_args(i), sync=True)
        return fp.get_state()
    finally:
        fp.close()


@pytest.mark.parametrize("path", ["fused", "plain"])
def test_single_tracer_matches_oracle(path):
    cfg = config.config1(nb=128)
    w, o, crp, cre = _inputs(cfg, 1, 601)
    g_crp, g_cre = _run(cfg, path, w, crp, cre, [12])
    o_crp, o_cre = crp.copy(), cre.copy()
    q = np.zeros_like(crp)
    o.snapshot(*w.snapshot_args(12), q, q, o_crp, o_cre, mass=w.mass)
    assert rel_err(g_cre, o_cre) <= 1e-10 and rel_err(g_crp, o_crp) <= 1e-10


@pytest.mark.parametrize("path,eta_cap", [("fused", 0.0), ("plain", 0.0), ("fused", 0.05)])
def test_chunked_workspace_equals_unchunked(path, eta_cap):
    cfg = dataclasses.replace(config.config1(nb=128), eta_dpp_cap=eta_cap)
    n = 37
    w, _, crp, cre = _inputs(cfg, n, 602)
    full = _run(cfg, path, w, crp, cre, [30, 31])
    # room for about five tracers' evolve workspace
    nseg = max(1, min(64, cfg.coeff_interp_max_segments))
    nseg_ws = 1 if path == "plain" else nseg
    per_tracer = 8.0 * cfg.nb * (2 * nseg_ws * 3 + 2 * nseg_ws) + nseg_ws * 112
    chunked = _run(cfg, path, w, crp, cre, [30, 31], limit=5.5 * per_tracer)
    assert np.array_equal(full[0], chunked[0]) and np.array_equal(full[1], chunked[1])


@pytest.mark.parametrize("path", ["fused", "plain"])
def test_zero_spectra_stay_zero(path):
    cfg = config.config1(nb=128)
    n = 9
    w, _, crp, cre = _inputs(cfg, n, 603)
    crp[2:5] = 0.0
    cre[2:5] = 0.0
    g_crp, g_cre = _run(cfg, path, w, crp, cre, [40, 41])
    assert np.all(np.isfinite(g_crp)) and np.all(np.isfinite(g_cre))
    assert not np.any(g_crp[2:5]) and not np.any(g_cre[2:5])
    assert np.any(g_cre[0]) and np.any(g_crp[0])


def test_invalid_calls_report_and_keep_the_context_usable():
    cfg = config.config1(nb=128)
    w, _, crp, cre = _inputs(cfg, 4, 604)
    fp = native.TracerFP(cfg, path="fused")
    try:
        # snapshot before any state
        with pytest.raises(native.CromaError, match="set_state"):
            fp.snapshot(*w.snapshot_args(5), sync=True)
        with pytest.raises(native.CromaError):
            fp.set_state(np.zeros((0, cfg.nb)), np.zeros((0, cfg.nb)))
        fp.set_state(crp, cre, mass=w.mass)
        bg0, bg1, z0, z1, allow, dt, el = w.snapshot_args(5)
        with pytest.raises(native.CromaError, match="dt_snap"):
            fp.snapshot(bg0, bg1, z0, z1, allow, 0.0, el, sync=True)
        with pytest.raises(native.CromaError, match="dt_snap"):
            fp.snapshot(bg0, bg1, z0, z1, allow, -1.0, el, sync=True)
        # still usable
        fp.snapshot(bg0, bg1, z0, z1, allow, dt, el, sync=True)
        g_crp, g_cre = fp.get_state()
        assert np.all(np.isfinite(g_cre)) and np.any(g_cre)
    finally:
        fp.close()
