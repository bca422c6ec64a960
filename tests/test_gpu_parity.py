"""GPU parity of the FP64 evolve paths (plain and fused) against the golden fixtures (outputs
of the reference's own CPU code) through the C ABI.

Bar: nsub, n_on and bucket ids bit-exact; spectra within 1e-10 relative
(on bins above 1e-12 of each tracer's peak), the reference's own CPU/CUDA
consistency tolerance (analysis/compare_tracer_outputs.py:126-127)."""
import numpy as np
import pytest

from conftest import load_package
from golden_io import Case, case_names, rel_err

load_package()
from croma_fp_b200 import native  # noqa: E402

SPECTRA_RTOL = 1e-10
pytestmark = pytest.mark.gpu


def _run_case(name, path):
    c = Case(name)
    d = c.d
    fp = native.TracerFP(c.cfg, path=path)
    fp.set_state(d["crp0"], d["cre0"], mass=d["mass"])
    results = []
    for k in range(c.nrun):
        fp.snapshot(*c.snapshot_args(k), sync=True)
        sched = fp.schedule()
        crp, cre = fp.get_state()
        results.append((sched, crp, cre))
    return c, fp, results


@pytest.mark.parametrize("path", ["plain", "fused"])
@pytest.mark.parametrize("name", case_names())
def test_path_matches_reference(name, path):
    c, fp, results = _run_case(name, path)
    d = c.d
    for k, (sched, crp, cre) in enumerate(results):
        assert np.array_equal(sched["nsub"], d[f"nsub_{k}"]), f"nsub mismatch at step {k}"
        assert np.array_equal(sched["non"], d[f"non_{k}"])
        assert np.array_equal(sched["bucket_ids"], d[f"bucket_ids_{k}"])
        e = rel_err(cre, d[f"cre_{k}"])
        assert e <= SPECTRA_RTOL, f"electron spectra rel err {e:.3e} at step {k}"
        if np.any(d[f"crp_{k}"]):
            e = rel_err(crp, d[f"crp_{k}"])
            assert e <= SPECTRA_RTOL, f"proton spectra rel err {e:.3e} at step {k}"


@pytest.mark.parametrize("name", ["c0_direct", "c1_asa256", "c4_asa512"])
def test_tables_match_reference(name):
    c = Case(name)
    d = c.d
    fp = native.TracerFP(c.cfg)
    gp, ge = fp.grid(0), fp.grid(1)
    assert np.array_equal(np.concatenate([gp[0], gp[1], gp[2], [gp[3], gp[4]]]), d["grid_p"])
    assert np.array_equal(np.concatenate([ge[0], ge[1], ge[2], [ge[3], ge[4]]]), d["grid_e"])
    row, m1, p1 = fp.ic_row(float(d["z"][c.isnap0]))
    ref = d["ic_row_0"]
    assert rel_err(np.concatenate([row, [m1, p1]])[None], ref[None], 0.0) <= 1e-12
    fqe, npmin = fp.secondary_kernel()
    assert np.array_equal(npmin, d["np_min_qe"])
    if "fqe" in d:
        assert rel_err(fqe, d["fqe"], 1e-30) <= 1e-12


FP32R_RTOL = 1e-6   # the precision form's bar: max relative error vs the FP64 reference


@pytest.mark.parametrize("name", case_names())
def test_fp32_refined_path_matches_reference(name):
    """The on-chip path with each sub-step solved in FP32 and refined once
    with an FP64 residual: schedule bit-exact (it is the same FP64 schedule),
    spectra within 1e-6 of the reference's FP64 result; the error is recorded
    per case."""
    c, fp, results = _run_case(name, "fp32r")
    d = c.d
    worst = 0.0
    for k, (sched, crp, cre) in enumerate(results):
        assert np.array_equal(sched["nsub"], d[f"nsub_{k}"])
        assert np.array_equal(sched["bucket_ids"], d[f"bucket_ids_{k}"])
        worst = max(worst, rel_err(cre, d[f"cre_{k}"]))
        if np.any(d[f"crp_{k}"]):
            worst = max(worst, rel_err(crp, d[f"crp_{k}"]))
    print(f"{name}: fp32-refined max rel err {worst:.3e}")
    assert worst <= FP32R_RTOL, f"fp32-refined spectra rel err {worst:.3e}"
