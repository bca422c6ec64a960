"""DSA injection on the GPU (croma_b200_dsa_inject) against the reference.

The golden fixtures golden_dsa_*.npz hold the reference's own results of
tracer_fp_apply_dsa_tracer_injection_snapshot for every shock form (raw
shock fields, merged-DSA fields), injection mode (tracer_state,
tracer_source) and reacceleration mode (off, positive_delta, drury83 with
its eta cap).  The GPU path runs on the resident spectra of a context of
either evolve path.  Its Simpson normalisation and
cumulative integrals are summed in a different order, so the bar is the
FP64 parity tolerance, 1e-10 relative; counts and flags are exact.  A DSA
injection followed by a snapshot is checked against the oracle doing the
same.
"""
import numpy as np
import pytest

from conftest import load_package
from golden_io import DSA_COMBOS, DsaCase, dsa_case_names, rel_err

load_package()
from croma_fp_b200 import config, native, synth  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-10


@pytest.mark.parametrize("path", ["fused", "plain"])
@pytest.mark.parametrize("name", dsa_case_names())
def test_dsa_inject_matches_reference(name, path):
    case = DsaCase(name)
    d = case.d
    fp = native.TracerFP(case.cfg, path=path)
    try:
        for merged, mode, reacc in DSA_COMBOS:
            exp = case.expected(merged, mode, reacc)
            fp.set_state(d["crp0"], d["cre0"], mass=d["mass"])
            fp.set_dsa(case.params(reacc))
            n = fp.dsa_inject(case.shocks(merged), 1.0, case.dt, mode, reacc)
            crp, cre = fp.get_state()
            qpi, qe, dis = fp.get_sources()
            tag = f"{name} {path} m{merged} mode{mode} r{reacc}"
            assert n == exp["ninj"], tag
            assert np.array_equal(dis, exp["dis"]), tag
            for got, key in ((crp, "crp"), (cre, "cre"), (qpi, "qpi"), (qe, "qepri")):
                if np.any(exp[key]):
                    assert rel_err(got, exp[key]) <= RTOL, f"{tag} {key}"
                else:
                    assert not np.any(got), f"{tag} {key}"
    finally:
        fp.close()


def test_dsa_then_snapshot_matches_oracle():
    """tracer_source injection then one snapshot (config 2's cadence: DSA on
    5% of tracer-snapshots), against the oracle doing the same."""
    import pyoracle
    cfg = config.config2()
    nt = 48
    w = synth.Workload(cfg, nt, 100, seed=91)
    isnap = 25
    args = w.snapshot_args(isnap)
    sh = synth.shocks(args[0], isnap, 91, fraction=0.25)
    prm = config.DsaParams()
    o = pyoracle.Oracle(cfg)
    gp, ge = o.grid(0), o.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    ocrp, ocre = crp.copy(), cre.copy()
    qpi, qe = np.zeros_like(crp), np.zeros_like(cre)
    dis = np.zeros(nt, np.uint8)
    n_or = o.dsa_inject(prm, sh, w.mass, 1.0, args[5], 2, 0, ocrp, ocre, qpi, qe, dis)
    o.snapshot(*args, qpi, qe, ocrp, ocre, mass=w.mass, dis=dis)
    fp = native.TracerFP(cfg, path="fused")
    try:
        fp.set_state(crp, cre, mass=w.mass)
        fp.set_dsa(prm)
        n_gpu = fp.dsa_inject(sh, 1.0, args[5], "tracer_source")
        fp.snapshot(*args)
        g_crp, g_cre = fp.get_state()
    finally:
        fp.close()
    assert n_gpu == n_or > 0
    assert rel_err(g_cre, ocre) <= RTOL
