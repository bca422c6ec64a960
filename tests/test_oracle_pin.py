"""Pins the CPU restatement (oracle/croma_oracle.c) against the reference.

Two anchors: the golden fixtures in tests/golden/ (produced by the
reference's own CPU code, see tests/golden/make_golden.py) and, where the
compiled reference oracle/_ref is present, a direct side-by-side run.
Integer outputs (nsub, n_on, bucket ids) must match exactly; the spectra
are compared at 1e-12 relative (they agree bit-for-bit with the same libm).
"""
import numpy as np
import pytest

import pyoracle
from golden_io import Case, case_names, rel_err

CASES = case_names()


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(name):
    c = Case(name)
    o = pyoracle.Oracle(c.cfg)
    d = c.d
    gp, ge = o.grid(0), o.grid(1)
    assert np.array_equal(np.concatenate([gp[0], gp[1], gp[2], [gp[3], gp[4]]]), d["grid_p"])
    assert np.array_equal(np.concatenate([ge[0], ge[1], ge[2], [ge[3], ge[4]]]), d["grid_e"])
    s, g, j = o.pp_cache()
    assert np.array_equal(s, d["sigma_pp"]) and np.array_equal(g, d["sigmoid_pp"]) and j == int(d["j_pp"])
    fqe, npmin = o.secondary_kernel()
    assert np.array_equal(npmin, d["np_min_qe"])
    if "fqe" in d:
        assert np.array_equal(fqe, d["fqe"])
    crp, cre = d["crp0"].copy(), d["cre0"].copy()
    q = np.zeros_like(crp)
    for k in range(c.nrun):
        args = c.snapshot_args(k)
        ic_cur = o.ic_row(args[2])
        assert np.array_equal(np.concatenate([ic_cur[0], [ic_cur[1], ic_cur[2]]]), d[f"ic_row_{k}"])
        nsub, non, bid, _ = o.snapshot(*args, q, np.zeros_like(cre), crp, cre, mass=d["mass"])
        assert np.array_equal(nsub, d[f"nsub_{k}"])
        assert np.array_equal(non, d[f"non_{k}"])
        assert np.array_equal(bid, d[f"bucket_ids_{k}"])
        assert rel_err(cre, d[f"cre_{k}"]) <= 1e-12
        if np.any(d[f"crp_{k}"]):
            assert rel_err(crp, d[f"crp_{k}"]) <= 1e-12


@pytest.mark.skipif(not pyoracle.reference_available(128), reason="oracle/_ref not built")
def test_oracle_cc_rows_match_reference():
    from croma_fp_b200 import config, synth
    cfg = config.config1(nb=128)
    o, r = pyoracle.Oracle(cfg), pyoracle.ReferenceCPU(cfg)
    w = synth.Workload(cfg, 24, 100, seed=5)
    bg = w.background(3)
    row, m1, p1 = o.ic_row(0.7)
    ric = np.repeat(row[:, None], 24, axis=1)
    a = o.cc_coeffs(1e-4, bg, ric, np.full(24, m1), np.full(24, p1), mass=w.mass)
    b = r.cc_coeffs(1e-4, bg, ric, np.full(24, m1), np.full(24, p1), mass=w.mass)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.skipif(not pyoracle.reference_available(128), reason="oracle/_ref not built")
def test_oracle_segment_windowed_matches_reference():
    from croma_fp_b200 import config, synth
    cfg = config.config1(nb=128, dpp_mode="ttd")
    o, r = pyoracle.Oracle(cfg), pyoracle.ReferenceCPU(cfg)
    nt = 16
    w = synth.Workload(cfg, nt, 100, seed=9)
    gp, ge = o.grid(0), o.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    crp2, cre2 = crp.copy(), cre.copy()
    bg = w.background(7)
    row, m1, p1 = o.ic_row(0.3)
    ric = np.repeat(row[:, None], nt, axis=1)
    rng = np.random.default_rng(3)
    qpi = rng.uniform(0, 1e40, crp.shape)
    qepri = rng.uniform(0, 1e40, cre.shape)
    dis = (np.arange(nt) % 3 == 0).astype(np.uint8)
    for args in ((7, 2e-4, True, 2, 5), (5, 1e-3, False, 0, 5)):
        o.evolve_segment(*args, bg, ric, np.full(nt, m1), np.full(nt, p1), qpi, qepri, crp, cre,
                         mass=w.mass, dis=dis)
        r.evolve_segment(*args, bg, ric, np.full(nt, m1), np.full(nt, p1), qpi, qepri, crp2, cre2,
                         mass=w.mass, dis=dis)
        assert np.array_equal(crp, crp2) and np.array_equal(cre, cre2)


@pytest.mark.skipif(not pyoracle.reference_available(128), reason="oracle/_ref not built")
def test_oracle_nsub_edge_inputs_match_reference():
    """Zero / negative divergence, zero-field and tiny-density tracers."""
    from croma_fp_b200 import config, synth
    cfg = config.config0(nsub_max=0, reacc_window_mode=1, f_eddy=0.05)
    o, r = pyoracle.Oracle(cfg), pyoracle.ReferenceCPU(cfg)
    bg = synth.background(64, 1, 77)
    bg[3, :8] = 0.0
    bg[3, 8:16] = -5.0
    bg[2, 16:24] = 0.0
    bg[0, 24:32] = 1e-9
    bg[5, 32:40] = 0.0
    row, _, _ = o.ic_row(0.0)
    for dt in (1e-3, 0.07, 3.0):
        a = o.nsub(dt, bg, row)
        b = r.nsub(dt, bg, row)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
