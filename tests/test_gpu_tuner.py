"""The steps-kernel autotuner (fused path): after the first snapshot each
evolving species has a tuned variant and a calibration time for every
admissible variant; CROMA_CUDA_TRIDIAG=pcr restricts it to warp PCR and
=thomas to the warp-scan variants, and whichever variant runs, the spectra
match the reference's (golden fixture) to the FP64 bar."""
import numpy as np
import pytest

from conftest import load_package
from golden_io import Case, rel_err

load_package()
from croma_fp_b200 import native  # noqa: E402

pytestmark = pytest.mark.gpu


def _run(name, env, monkeypatch):
    if env is None:
        monkeypatch.delenv("CROMA_CUDA_TRIDIAG", raising=False)
    else:
        monkeypatch.setenv("CROMA_CUDA_TRIDIAG", env)
    c = Case(name)
    d = c.d
    fp = native.TracerFP(c.cfg, path="fused")
    try:
        fp.set_state(d["crp0"], d["cre0"], mass=d["mass"])
        fp.snapshot(*c.snapshot_args(0), sync=True)
        crp, cre = fp.get_state()
        tunes = [fp.tuning(s) for s in (0, 1)]
    finally:
        fp.close()
    assert rel_err(cre, d["cre_0"]) <= 1e-10
    if np.any(d["crp_0"]):
        assert rel_err(crp, d["crp_0"]) <= 1e-10
    return tunes


@pytest.mark.parametrize("name", ["c1_asa128", "c4_asa512"])
def test_tuner_chooses_and_records(name, monkeypatch):
    tunes = _run(name, None, monkeypatch)
    for t in tunes:
        assert t["tuned"] == 1
        ms = t["variant_ms"]
        assert all(v is not None and v > 0 for v in ms.values()), ms
        chosen = {("thomas-scan", 1): "scan x1", ("thomas-scan", 2): "scan x2",
                  ("thomas-scan-smem", 1): "smem scan x1", ("thomas-scan-smem", 2): "smem scan x2",
                  ("pcr", 1): "pcr x1"}[(t["solver"], t["warps_per_block"])]
        assert ms[chosen] == min(ms.values())
    print(name, tunes)


@pytest.mark.parametrize("env,solver", [("pcr", "pcr"), ("thomas", "thomas-scan")])
def test_tridiag_env_restricts_the_tuner(env, solver, monkeypatch):
    for t in _run("c1_asa128", env, monkeypatch):
        assert t["tuned"] == 1 and t["solver"].startswith(solver)
        if env == "pcr":
            assert t["variant_ms"]["scan x1"] is None
        else:
            assert t["variant_ms"]["pcr x1"] is None


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("name", ["c1_asa256", "c4_asa512"])
def test_every_steps_variant_matches_reference(name, variant, monkeypatch):
    monkeypatch.setenv("CROMA_B200_STEPS_VARIANT", str(variant))
    _run(name, None, monkeypatch)
