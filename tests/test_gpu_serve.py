"""Request serving (include/croma_b200_serve.h) on the GPU.

Requests of different sizes, species and snapshot counts run concurrently
on their own streams; each result must equal the oracle advancing the same
tracers through the same snapshots (FP64 parity, 1e-10).  Also checked:
admission refuses a request larger than the whole budget, a queued request
can be cancelled, strided backgrounds are read correctly, and the latency
statistics are filled.
"""
import numpy as np
import pytest

from conftest import load_package
from golden_io import rel_err

load_package()
from croma_fp_b200 import config, serve, synth  # noqa: E402

pytestmark = pytest.mark.gpu
# seed species -> the mask the reference's semantics needs (protons feed
# secondary electrons, so a proton seed evolves both species)
SEEDS = [("electron_proton", 3), ("electron_only", 2), ("proton_only", 3), ("electron_proton", 3),
         ("electron_only", 2)]


def _inputs(cfg, n, nsnap, seed, first):
    w = synth.Workload(cfg, n, 100, seed=seed)
    bg = np.stack([w.background(first + k) for k in range(nsnap + 1)])
    return w, bg, w.z[first:first + nsnap + 1].copy(), w.dt[first:first + nsnap].copy()


def _oracle(cfg, w, bg, z, dt, crp, cre, first):
    import pyoracle
    o = pyoracle.Oracle(cfg)
    for k in range(dt.size):
        o.snapshot(bg[k], bg[k + 1], float(z[k]), float(z[k + 1]), True, float(dt[k]),
                   float(w.elapsed[first + k]), np.zeros_like(crp), np.zeros_like(cre), crp, cre,
                   mass=w.mass)
    return crp, cre


def test_server_requests_match_oracle():
    base = config.config1(nb=128)
    srv = serve.Server(base, hbm_budget_gb=20.0, max_concurrent=3, workspace_gb_per_request=0.5)
    try:
        jobs = []
        for i, (n, nsnap) in enumerate([(40, 2), (17, 3), (64, 2), (33, 1), (8, 2)]):
            seed, mask = SEEDS[i]
            cfg = config.config1(nb=128, species=seed)
            assert cfg.species_mask() == mask
            first = 10 + 7 * i
            w, bg, z, dt = _inputs(cfg, n, nsnap, 500 + i, first)
            import pyoracle
            o = pyoracle.Oracle(cfg)
            gp, ge = o.grid(0), o.grid(1)
            crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
            rid = srv.submit(bg, z, dt, crp, cre, mass=w.mass, species_mask=mask,
                             elapsed0=float(w.elapsed[first]))
            jobs.append((rid, cfg, w, bg, z, dt, crp.copy(), cre.copy(), first))
        for rid, cfg, w, bg, z, dt, crp, cre, first in jobs:
            assert srv.wait(rid, 300.0) == serve.DONE, srv.result(rid)
            rc, lat, run, msg = srv.result(rid)
            assert rc == 0 and lat >= run > 0.0, msg
            g_crp, g_cre = srv.output(rid)
            o_crp, o_cre = _oracle(cfg, w, bg, z, dt, crp, cre, first)
            if np.any(o_cre):
                assert rel_err(g_cre, o_cre) <= 1e-10
            if np.any(o_crp):
                assert rel_err(g_crp, o_crp) <= 1e-10
        st = srv.stats()
        assert st["completed"] == len(jobs) and st["queued"] == 0 and st["running"] == 0
        assert 0.0 < st["p50_s"] <= st["p99_s"]
    finally:
        srv.close()


def test_server_budget_cancel_and_strides():
    base = config.config1(nb=128)
    srv = serve.Server(base, hbm_budget_gb=2.0, max_concurrent=1, workspace_gb_per_request=0.25)
    try:
        big = int(4.0e9 / (5 * 128 * 8))
        assert srv.request_bytes(big) > 2.0e9
        cfg = config.config1(nb=128, species="electron_only")
        w, bg, z, dt = _inputs(cfg, 16, 2, 7, 30)
        with pytest.raises(serve.ServeError):
            srv.submit(np.zeros((3, 8, big)), z, dt, ntracer=big)
        # one runner: the first request runs, the second waits and is cancelled
        w2, bg2, z2, dt2 = _inputs(cfg, 256, 6, 8, 20)
        first = srv.submit(bg2, z2, dt2, species_mask=2)
        second = srv.submit(bg2, z2, dt2, species_mask=2)
        assert srv.cancel(second) == 0
        assert srv.wait(second, 60.0) == serve.CANCELLED
        assert srv.wait(first, 300.0) == serve.DONE
        srv.forget(second)
        srv.output(first)
        # strided view into a wider background pool: tracers 5..20 of 32
        wp, pool, zp, dtp = _inputs(cfg, 32, 2, 9, 40)
        sub = np.ascontiguousarray(pool[:, :, 5:21])
        import pyoracle
        o = pyoracle.Oracle(cfg)
        gp, ge = o.grid(0), o.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 16, cfg.species)
        flat = pool.reshape(-1)
        rid = srv.submit(flat[5:], zp, dtp, crp, cre, species_mask=2, field_stride=32, snap_stride=8 * 32,
                         ntracer=16, elapsed0=float(wp.elapsed[40]))
        assert srv.wait(rid, 300.0) == serve.DONE
        g_crp, g_cre = srv.output(rid)
        wsub = synth.Workload(cfg, 16, 100, seed=9)
        _, o_cre = _oracle(cfg, wsub, sub, zp, dtp, crp, cre, 40)
        assert rel_err(g_cre, o_cre) <= 1e-10
    finally:
        srv.close()


@pytest.mark.parametrize("path", ["fused", "fp32r"])
def test_result_alone_equals_result_in_the_mix_256_bins(path):
    """Config 3's mix at 256 bins with all three seed species: requests that
    run concurrently (admitted as slots free up, their kernels overlapping on
    the device) give the same spectra as each request run alone, within the
    FP64 bar 1e-10 (they are computed by the same kernels on their own
    contexts, so in practice bit for bit)."""
    base = config.config1(nb=256)
    specs = [(48, 3, "electron_only", 2), (20, 2, "proton_only", 3), (64, 2, "electron_proton", 3),
             (33, 4, "electron_only", 2), (16, 3, "proton_only", 3), (40, 3, "electron_proton", 3)]
    reqs = []
    for i, (n, nsnap, seed, mask) in enumerate(specs):
        cfg = config.config1(nb=256, species=seed)
        first = 12 + 5 * i
        w, bg, z, dt = _inputs(cfg, n, nsnap, 900 + i, first)
        import pyoracle
        o = pyoracle.Oracle(cfg)
        gp, ge = o.grid(0), o.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        reqs.append(dict(bg=bg, z=z, dt=dt, crp=crp, cre=cre, mass=w.mass, mask=mask, e0=float(w.elapsed[first])))

    def submit(srv, r):
        return srv.submit(r["bg"], r["z"], r["dt"], r["crp"], r["cre"], mass=r["mass"], species_mask=r["mask"],
                          elapsed0=r["e0"])

    mix = []
    srv = serve.Server(base, hbm_budget_gb=20.0, max_concurrent=4, workspace_gb_per_request=0.5, path=path)
    try:
        ids = [submit(srv, r) for r in reqs]
        for rid in ids:
            assert srv.wait(rid, 300.0) == serve.DONE, srv.result(rid)
            mix.append(srv.output(rid))
        assert srv.stats()["completed"] == len(reqs)
    finally:
        srv.close()
    srv = serve.Server(base, hbm_budget_gb=20.0, max_concurrent=1, workspace_gb_per_request=0.5, path=path)
    try:
        for r, (m_crp, m_cre) in zip(reqs, mix):
            rid = submit(srv, r)
            assert srv.wait(rid, 300.0) == serve.DONE, srv.result(rid)
            a_crp, a_cre = srv.output(rid)
            for alone, inmix in ((a_crp, m_crp), (a_cre, m_cre)):
                if np.any(alone):
                    assert rel_err(inmix, alone) <= 1e-10
                else:
                    assert not np.any(inmix)
    finally:
        srv.close()
