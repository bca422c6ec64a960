"""IC emissivity: prepare_ic_emission_cuda_batch against the reference.

The fixture golden_emission_ic.npz holds the reference's own kernel table
(prepare_ic_kernel_flat, src/fp_shared_core.c:1780-1807) and emissivities
(prepare_ic_emission_batch, :2131-2164) for 128- and 256-bin electron
spectra.  The CPU test pins the restatement (a sum over electron bins of
fic x N x dp) on the fixture; the GPU test runs the library's entry point on
the same inputs.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import load_package
from golden_io import GOLDEN_DIR, rel_err

load_package()
from croma_fp_b200 import ref_abi  # noqa: E402

FIX = np.load(os.path.join(GOLDEN_DIR, "golden_emission_ic.npz"))


@pytest.mark.parametrize("nb", [128, 256])
def test_ic_emission_restatement_matches_reference(nb):
    cre, fic, eps, dp = (FIX[f"nb{nb}_{k}"] for k in ("cre", "fic", "eps", "dp"))
    mine = np.array([[np.sum(f * row * dp) for f in fic] for row in cre])
    assert rel_err(mine, eps) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("nb", [128, 256])
def test_ic_emission_gpu_matches_reference(nb):
    cre, fic, eps, dp = (FIX[f"nb{nb}_{k}"] for k in ("cre", "fic", "eps", "dp"))
    abi = ref_abi.RefAbi(nb)
    lib = abi.lib
    lib.prepare_ic_emission_cuda_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    inp = ref_abi.FpIcEmissionBatchInput(cre.shape[0], fic.shape[0], float(FIX["z"]), float(FIX["nu_min"]),
                                         float(FIX["nu_max"]), ref_abi.dptr(cre), ref_abi.dptr(fic))
    p = np.geomspace(1.0, 10.0, nb)   # only dp is read
    cg = abi.grid(p, np.ascontiguousarray(dp), p, p[0] * 0.9, p[-1] * 1.1)
    out = np.empty_like(eps)
    ms = C.c_double()
    rc = lib.prepare_ic_emission_cuda_batch(C.byref(inp), C.byref(cg), ref_abi.dptr(out), C.byref(ms))
    assert rc == 0, abi.error()
    assert rel_err(out, eps) <= 1e-12
