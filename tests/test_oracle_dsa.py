"""Pins the DSA-injection restatement (oracle/croma_oracle_dsa.c) against the
reference's tracer_fp_apply_dsa_tracer_injection_snapshot.

Anchors: the golden fixtures golden_dsa_*.npz (written by the reference's own
CPU code, tests/golden/make_golden.py) for every shock form (raw shock fields
and merged-DSA fields), injection mode (tracer_state, tracer_source) and
reacceleration mode (off, positive_delta, drury83 with its eta cap), plus a
direct side-by-side run where oracle/_ref is present.  The restatement uses
the reference's operation order, so the bar is 1e-13 relative.
"""
import numpy as np
import pytest

import pyoracle
from golden_io import DSA_COMBOS, DsaCase, dsa_case_names, rel_err
from conftest import load_package

load_package()
from croma_fp_b200 import config, synth  # noqa: E402


def _run(impl, case, merged, mode, reacc):
    d = case.d
    crp, cre = d["crp0"].copy(), d["cre0"].copy()
    qpi, qe = np.zeros_like(crp), np.zeros_like(cre)
    dis = np.zeros(case.ntracer, np.uint8)
    n = impl.dsa_inject(case.params(reacc), case.shocks(merged), d["mass"], 1.0, case.dt, mode, reacc,
                        crp, cre, qpi, qe, dis)
    return dict(crp=crp, cre=cre, qpi=qpi, qepri=qe, dis=dis, ninj=n)


def _check(got, exp, tol):
    assert got["ninj"] == exp["ninj"]
    assert np.array_equal(got["dis"], exp["dis"])
    for k in ("crp", "cre", "qpi", "qepri"):
        if np.any(exp[k]):
            assert rel_err(got[k], exp[k]) <= tol, k
        else:
            assert not np.any(got[k]), k


@pytest.mark.parametrize("name", dsa_case_names())
@pytest.mark.parametrize("combo", DSA_COMBOS, ids=lambda c: f"m{c[0]}_mode{c[1]}_r{c[2]}")
def test_dsa_oracle_matches_golden(name, combo):
    case = DsaCase(name)
    o = pyoracle.Oracle(case.cfg)
    got = _run(o, case, *combo)
    _check(got, case.expected(*combo), 1e-13)
    if combo[2] == 0 and combo[1] == 1:
        # fresh injection happened somewhere and left the unshocked tracers alone
        assert got["ninj"] > 0
        untouched = np.all(got["crp"] == case.d["crp0"], axis=1)
        assert untouched.sum() >= case.ntracer - got["ninj"]


@pytest.mark.skipif(not pyoracle.reference_available(128), reason="oracle/_ref not built")
def test_dsa_oracle_matches_reference_other_params():
    """Parameters away from the defaults: another efficiency model, one
    species, a nonzero upstream speed and pre-shock density override."""
    cfg = config.config1(nb=128)
    w = synth.Workload(cfg, 40, 100, seed=77)
    bg = w.background(30)
    sh = synth.shocks(bg, 30, 77, fraction=0.5)
    sh["upstream_speed_cgs"] = np.where(sh["mach"] > 0, 3.0e8, 0.0)
    sh["pre_density_cgs"] = np.where(np.arange(40) % 3 == 0, bg[0] * 1.0e-24, 0.0)
    for model, species in ((2, 0), (0, 2), (4, 1)):
        prm = config.DsaParams(eta_model_initial=model, eta_model_reacc=model + 1, inject_species=species)
        res = []
        for impl in (pyoracle.Oracle(cfg), pyoracle.ReferenceCPU(cfg)):
            gp, ge = impl.grid(0), impl.grid(1)
            crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 40, cfg.species)
            crp *= 1e3
            qpi, qe = np.zeros_like(crp), np.zeros_like(cre)
            dis = np.zeros(40, np.uint8)
            n = impl.dsa_inject(prm, sh, w.mass, 1.0, float(w.dt[30]), 1, 1, crp, cre, qpi, qe, dis)
            res.append(dict(crp=crp, cre=cre, qpi=qpi, qepri=qe, dis=dis, ninj=n))
        _check(res[0], res[1], 1e-13)
