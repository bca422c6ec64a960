"""The drop-in boundary checked by a C compiler: every struct of
include/fp_cuda_backend.h (CRspectrum, FpCoeffBatchInput, the emission
inputs, FpChangCooperSolveBatchInput, FpCudaOutputSchedule,
FpCudaPipelineInput, FpCudaPipelineTimes) has the size, field offsets and
field sizes that the reference's own headers give
(include/fp_cuda_backend.h:12-90, include/fp_shared_core.h:366-690,
include/params.h:52-61 of kosukenishiwaki/croma-fp), at np = npe = 128, 256
and 512.  The reference's figures are committed in
tests/golden/abi_layout_ref.json (tests/golden/make_abi_layout.py); where
the reference checkout is present they are measured again live."""
import json
import os

import pytest

from abi_layout import NBS, ROOT, measure, struct_fields

FIX = json.load(open(os.path.join(ROOT, "tests", "golden", "abi_layout_ref.json")))


@pytest.mark.parametrize("nb", NBS)
def test_struct_layouts_match_reference_headers(nb):
    ours = measure(os.path.join(ROOT, "include"), nb)
    ref = FIX[str(nb)]
    assert set(ours) == set(ref)
    bad = {k: (ours[k], ref[k]) for k in ref if ours[k] != ref[k]}
    assert not bad, bad


def test_every_reference_struct_field_is_covered():
    """The field lists come from this repository's header; a field the
    reference has and this header lacks changes the struct's size, which the
    layout test compares, and every struct the ABI passes is covered."""
    names = [n for n, _ in struct_fields()]
    for n in ("CRspectrum", "FpCoeffBatchInput", "FpSynchEmissionBatchInput", "FpGammaEmissionBatchInput",
              "FpNeutrinoEmissionBatchInput", "FpChangCooperSolveBatchInput", "FpCudaOutputSchedule",
              "FpCudaPipelineInput", "FpCudaPipelineTimes"):
        assert n in names


REF = os.environ.get("CROMA_REFERENCE_ROOT", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include")), reason="reference checkout not present")
@pytest.mark.parametrize("nb", NBS)
def test_struct_layouts_live_against_reference_checkout(nb):
    assert measure(os.path.join(REF, "include"), nb) == measure(os.path.join(ROOT, "include"), nb)
