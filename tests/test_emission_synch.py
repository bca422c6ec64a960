"""Synchrotron emission: the pitch-kernel table and both branches of the
emissivity (src/fp_shared_core.c:2008-2129, src/Synchrotron.c:62-103).

golden_emission_synch.npz holds the reference's own results on one set of
tables (tests/golden/make_golden.py, make_synch_emission): the pitch-kernel
table, the emissivity through the table and through the pitch-angle loop.
The numpy restatement in oracle/pyoracle.py is pinned to them on the CPU;
the device entry points prepare_synch_pitch_kernel_table_cuda and
prepare_synch_emission_cuda_batch (with and without a table) are checked
against them on the GPU.  pow / log differ from the host's by an ulp and
the device sums the bins of a frequency in another order: bar 1e-12
relative.
"""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from conftest import load_package

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
import pyoracle  # noqa: E402

RTOL = 1e-12


def _golden():
    return np.load(os.path.join(HERE, "golden", "golden_emission_synch.npz"))


def _rel(x, y):
    y = np.asarray(y)
    m = np.abs(y) > 0
    assert np.all(x[~m] == 0.0)
    return float(np.max(np.abs(x - y)[m] / np.abs(y)[m])) if m.any() else 0.0


def test_restatement_matches_reference_synch():
    d = _golden()
    t = pyoracle.synch_pitch_table(d["logy"], d["w"], float(d["logb_min"]), float(d["inv_dlogb"]),
                                   int(d["nlogb"]), float(d["xmin"]), d["logx"], d["logfx"], d["fx"])
    assert _rel(t, d["table"]) <= RTOL
    e = pyoracle.synch_emission_theta(d["cre"], d["dp"], d["b_dyn"], d["logb"], d["logy"], d["w"],
                                      float(d["xmin"]), d["logx"], d["logfx"], d["fx"])
    assert _rel(e, d["eps_theta"]) <= RTOL
    # the cut-off rows stop at the first je whose N[je+1] is zero, and a
    # spectrum zero from bin 3 emits nothing
    assert d["eps_theta"][2].max() == 0.0 and d["eps_theta"][0, 0] > 0.0


def _synch_input(abi, ref_abi, d, keep):
    nfreq, nb, nth = d["logy"].shape
    sin = ref_abi.FpSynchEmissionBatchInput()
    sin.ncell, sin.nfreq = d["cre"].shape[0], nfreq
    sin.nx_tab, sin.ntheta_pitch = len(d["logx"]), nth
    sin.xmin = float(d["xmin"])
    for name in ("fx", "logfx", "logx", "w", "b_dyn", "logb", "cre"):
        keep[name] = np.ascontiguousarray(d[name], dtype=np.float64)
    sin.fx_tab, sin.logfx_tab, sin.logx_tab = (ref_abi.dptr(keep["fx"]), ref_abi.dptr(keep["logfx"]),
                                               ref_abi.dptr(keep["logx"]))
    sin.pitch_weight = ref_abi.dptr(keep["w"])
    sin.b_dyn, sin.logb, sin.cre_batch = ref_abi.dptr(keep["b_dyn"]), ref_abi.dptr(keep["logb"]), \
        ref_abi.dptr(keep["cre"])
    # logy as the reference's [nfreq][npe] pointer view of [ntheta] rows
    logy = np.ascontiguousarray(d["logy"], dtype=np.float64)
    rows = (C.POINTER(C.c_double) * (nfreq * nb))()
    for nf in range(nfreq):
        for je in range(nb):
            rows[nf * nb + je] = logy[nf, je].ctypes.data_as(C.POINTER(C.c_double))
    planes = (C.POINTER(C.POINTER(C.c_double)) * nfreq)()
    for nf in range(nfreq):
        planes[nf] = C.cast(C.byref(rows, nf * nb * C.sizeof(C.POINTER(C.c_double))),
                            C.POINTER(C.POINTER(C.c_double)))
    keep["logy"], keep["rows"], keep["planes"] = logy, rows, planes
    sin.logy = C.cast(planes, C.c_void_p).value
    return sin


@pytest.mark.gpu
def test_gpu_synch_table_and_emission_match_reference():
    load_package()
    from croma_fp_b200 import ref_abi
    d = _golden()
    abi = ref_abi.RefAbi(int(d["nb"]))
    keep = {}
    sin = _synch_input(abi, ref_abi, d, keep)
    ms = C.c_double()
    # the pitch-kernel table on the device
    nlogb = int(d["nlogb"])
    sin.nlogb, sin.logb_min, sin.inv_dlogb = nlogb, float(d["logb_min"]), float(d["inv_dlogb"])
    table = np.empty_like(d["table"])
    assert abi.lib.prepare_synch_pitch_kernel_table_cuda(C.byref(sin), ref_abi.dptr(table), C.byref(ms)) == 0, \
        abi.error()
    assert _rel(table, d["table"]) <= RTOL
    nb = int(d["nb"])
    grid = abi.grid(np.zeros(nb), d["dp"], np.zeros(nb), 0.0, 0.0)
    # emissivity through the table
    sin.pitch_kernel_table = ref_abi.dptr(table)
    out = np.empty_like(d["eps_table"])
    assert abi.lib.prepare_synch_emission_cuda_batch(C.byref(sin), C.byref(grid), ref_abi.dptr(out),
                                                     C.byref(ms)) == 0, abi.error()
    assert _rel(out, d["eps_table"]) <= RTOL
    # and without it: the pitch-angle loop
    sin.pitch_kernel_table = None
    sin.nlogb = 0
    out = np.empty_like(d["eps_theta"])
    assert abi.lib.prepare_synch_emission_cuda_batch(C.byref(sin), C.byref(grid), ref_abi.dptr(out),
                                                     C.byref(ms)) == 0, abi.error()
    assert _rel(out, d["eps_theta"]) <= RTOL
