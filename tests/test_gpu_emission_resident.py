"""Emissivities of a context's resident spectra (croma_b200_emission_*).

The resident entry points run the reference-ABI emission kernels on the
spectra the context holds on the device, so their results must equal the
reference-ABI calls (prepare_ic/gamma/neutrino/synch_emission_cuda_batch, which
are themselves checked against the reference's CPU code in
test_emission_ic.py, test_emission_synch.py and test_gpu_ref_abi.py) on the
same spectra bit for bit: right after set_state and after a snapshot has
evolved them.  Calls without resident state or with mis-shaped tables fail
with an error and leave the context usable.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_package

load_package()
from croma_fp_b200 import config, native, ref_abi, synth  # noqa: E402

pytestmark = pytest.mark.gpu


def _ref_call(abi, fn, inp, grid, out):
    ms = C.c_double()
    assert fn(C.byref(inp), C.byref(grid), ref_abi.dptr(out), C.byref(ms)) == 0, abi.error()
    return out


def _reference(abi, gp, ge, crp, cre, fic, kern, n_gas, beta_p, table, b_dyn, logb, tab_args):
    n = crp.shape[0]
    L = abi.lib
    L.prepare_ic_emission_cuda_batch.argtypes = [C.c_void_p] * 4
    cg_p, cg_e = abi.grid(*gp), abi.grid(*ge)
    crp, cre = np.ascontiguousarray(crp), np.ascontiguousarray(cre)
    ic = ref_abi.FpIcEmissionBatchInput(n, fic.shape[0], 0.1, 8.0, 20.0, ref_abi.dptr(cre), ref_abi.dptr(fic))
    e_ic = _ref_call(abi, L.prepare_ic_emission_cuda_batch, ic, cg_e, np.empty((n, fic.shape[0])))
    had = ref_abi.FpHadronicEmissionBatchInput(n, kern.shape[0], 0.1, -1.0, 3.0, ref_abi.dptr(n_gas),
                                               ref_abi.dptr(crp), ref_abi.dptr(beta_p), ref_abi.dptr(kern))
    e_ga = _ref_call(abi, L.prepare_gamma_emission_cuda_batch, had, cg_p, np.empty((n, kern.shape[0])))
    sin = ref_abi.FpSynchEmissionBatchInput()
    sin.ncell, sin.nfreq, sin.nlogb = n, table.shape[1], table.shape[0]
    sin.logb_min, sin.inv_dlogb = tab_args
    sin.pitch_kernel_table = ref_abi.dptr(table)
    sin.b_dyn, sin.logb, sin.cre_batch = ref_abi.dptr(b_dyn), ref_abi.dptr(logb), ref_abi.dptr(cre)
    e_sy = _ref_call(abi, L.prepare_synch_emission_cuda_batch, sin, cg_e, np.empty((n, table.shape[1])))
    return e_ic, e_ga, e_sy


@pytest.mark.parametrize("nb", [128, 256])
def test_resident_emission_equals_reference_abi(nb):
    cfg = config.config1(nb=nb)
    n = 301
    w = synth.Workload(cfg, n, 100, seed=811)
    rng = np.random.default_rng(812)
    fp = native.TracerFP(cfg, path="fused")
    try:
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        crp *= rng.uniform(0.5, 2.0, (n, 1))
        cre[5, nb // 2:] = 0.0        # a cut-off spectrum: the synchrotron sum stops early
        bg = w.background(30)
        n_gas, b_dyn = np.ascontiguousarray(bg[0]), np.ascontiguousarray(bg[2])
        logb = np.ascontiguousarray(np.log10(b_dyn))
        beta_p = np.ascontiguousarray(gp[0] / np.sqrt(1.0 + gp[0] ** 2))
        fic = np.ascontiguousarray(rng.uniform(1e-3, 1.0, (7, nb)))
        kern = np.ascontiguousarray(rng.uniform(1e-3, 1.0, (9, nb)))
        table = np.ascontiguousarray(rng.uniform(1e-3, 1.0, (16, 5, nb)))
        table[4, :, 10:20] = 0.0      # zero entries: the linear branch of the log-K interpolation
        tab_args = (-9.0, 16 / 5.0)
        abi = ref_abi.RefAbi(nb)

        fp.set_state(crp, cre, mass=w.mass)
        for k in range(2):
            if k == 1:
                fp.snapshot(*w.snapshot_args(30), sync=True)
            s_crp, s_cre = fp.get_state()
            want = _reference(abi, gp, ge, s_crp, s_cre, fic, kern, n_gas, beta_p, table, b_dyn, logb, tab_args)
            e_ic, ms = fp.emission_ic(fic)
            assert ms > 0.0
            e_ga, _ = fp.emission_hadronic(kern, n_gas, beta_p, -1.0, 3.0)
            e_sy, _ = fp.emission_synch(table, b_dyn, logb, *tab_args)
            for got, ref in zip((e_ic, e_ga, e_sy), want):
                assert got.shape == ref.shape
                assert np.array_equal(got, ref)
            assert np.any(e_ic > 0) and np.any(e_ga > 0) and np.any(e_sy > 0)
    finally:
        fp.close()


def test_resident_emission_errors_keep_the_context_usable():
    cfg = config.config1(nb=128)
    fp = native.TracerFP(cfg, path="fused")
    try:
        fic = np.ones((3, cfg.nb))
        with pytest.raises(native.CromaError, match="set_state"):
            fp.emission_ic(fic)
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 40, cfg.species)
        fp.set_state(crp, cre)
        with pytest.raises(ValueError):
            fp.emission_ic(np.ones((3, cfg.nb + 1)))
        with pytest.raises(native.CromaError, match="pitch-kernel table"):
            fp.emission_synch(np.ones((1, 2, cfg.nb)), np.full(40, 1e-6), np.full(40, -6.0), -9.0, 1.0)
        eps, _ = fp.emission_ic(fic)
        assert eps.shape == (40, 3) and np.all(np.isfinite(eps)) and np.any(eps > 0)
    finally:
        fp.close()
