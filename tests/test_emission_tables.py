"""Emission kernel tables and the resident emission, against the reference.

The fixture golden_emission_tables.npz (tests/golden/make_golden.py) holds
the reference's own gamma / neutrino / IC kernel tables
(prepare_*_kernel_flat, src/fp_shared_core.c:1724-1807), its synchrotron
tables (tracer_fp_synch_data_init_tables and the pitch-kernel table of
tracer_fp_refresh_synch_kernel_table, src/tracer_fp_synch.c) and its
emissivities (prepare_*_emission_cell_major) on 128-bin spectra, with the
config-4 band grids.

The synchrotron function F(x) = x int_x^inf K_5/3 comes from GNU GSL in the
reference, which is absent here; the checker restates it from the integral
definition (oracle/synch_fx.c).  The CPU tests pin that restatement to an
independent multiprecision Bessel-function quadrature and to the small- and
large-x asymptotes, and pin the emission sums (a numpy restatement of
Q_one and the IC / synchrotron sums) to the fixture.  The GPU tests compare
the device-built tables and the resident emission with the fixture.
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT, load_package
from golden_io import GOLDEN_DIR

load_package()
from croma_fp_b200 import config, native, ref_abi  # noqa: E402

FIX = np.load(os.path.join(GOLDEN_DIR, "golden_emission_tables.npz"))
PRM = json.loads(str(FIX["params"]))


def oracle_fx():
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    lib.oracle_synch_fx.restype = C.c_double
    lib.oracle_synch_fx.argtypes = [C.c_double]
    return lib.oracle_synch_fx


def rel_to_max(a, b):
    """Largest |a - b| over the entries of b above 1e-12 of max|b|, relative
    to each entry."""
    m = np.abs(b) > 1e-12 * np.max(np.abs(b))
    return float(np.max(np.abs(a - b)[m] / np.abs(b)[m])) if m.any() else 0.0


# ---------------------------------------------------------------- CPU
def test_synch_fx_restatement_matches_bessel_quadrature():
    mp = pytest.importorskip("mpmath")
    mp.mp.dps = 30
    F = oracle_fx()
    for x in (1e-20, 1e-10, 1e-4, 1e-2, 0.1, 0.29, 1.0, 3.0, 10.0, 30.0):
        X = mp.mpf(x)
        pts = sorted({X, *[p for p in (2 * X, 10 * X, 100 * X, mp.mpf(1), mp.mpf(10), mp.mpf(100)) if p > X]})
        ref = float(X * mp.quad(lambda s: mp.besselk(mp.mpf(5) / 3, s), pts + [mp.inf]))
        assert abs(F(x) / ref - 1.0) <= 1e-13, x


def test_synch_fx_restatement_asymptotes():
    F = oracle_fx()
    a = 4.0 * math.pi / (math.sqrt(3.0) * math.gamma(1.0 / 3.0))
    for x in (1e-25, 1e-23):   # F ~ a (x/2)^(1/3), next term O(x^(2/3))
        assert abs(F(x) / (a * (x / 2.0) ** (1.0 / 3.0)) - 1.0) <= 1e-13
    for x in (200.0, 300.0):   # F ~ sqrt(pi x / 2) e^-x (1 + 55 / (72 x))
        lead = math.sqrt(0.5 * math.pi * x) * math.exp(-x) * (1.0 + 55.0 / (72.0 * x))
        assert abs(F(x) / lead - 1.0) <= 2.0 / x ** 2


def test_synch_fx_table_in_fixture_is_the_restatement():
    F = oracle_fx()
    logx, logfx = FIX["syn_logx"], FIX["syn_logfx"]
    for i in range(0, len(logx), 97):
        x = 10.0 ** logx[i]
        want = math.log10(F(x)) if x <= 300.0 else math.log10(math.sqrt(0.5 * math.pi) * math.exp(-x) * x ** 0.5)
        assert abs(logfx[i] - want) <= 1e-14 * max(1.0, abs(want))


def test_emission_sums_restatement_matches_reference():
    """Q_one (trapezoid of beta N K dp, src/EMISSION.c:297-308) times E n_gas
    for gamma / neutrino, sum fic N dp for IC."""
    nbins = PRM["nbins"]
    beta = FIX["p_p"] / np.sqrt(1.0 + FIX["p_p"] ** 2)
    for kind, lo, hi in (("gamma", *PRM["egamma"]), ("nu", *PRM["enu"])):
        K = FIX["fga" if kind == "gamma" else "fnu"]
        d = (hi - lo) / nbins
        E = 10.0 ** (lo + d * np.arange(nbins))
        f = beta[None, None, :] * FIX["crp"][:, None, :] * K[None, :, :]
        q = 0.5 * np.sum((f[:, :, :-1] + f[:, :, 1:]) * FIX["dp_p"][None, None, 1:], axis=2)
        mine = E[None, :] * q * FIX["n_gas"][:, None]
        assert rel_to_max(mine, FIX[f"eps_{kind}"]) <= 1e-12
    mine = np.einsum("kj,cj,j->ck", FIX["fic"], FIX["cre"], FIX["dp_e"])
    assert rel_to_max(mine, FIX["eps_ic"]) <= 1e-12


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_device_kernel_tables_match_reference():
    nb, nbins = PRM["nb"], PRM["nbins"]
    abi = ref_abi.RefAbi(nb)
    L = abi.lib
    D = C.POINTER(C.c_double)
    for fn in ("prepare_gamma_kernel_flat_cuda", "prepare_neutrino_kernel_flat_cuda"):
        getattr(L, fn).argtypes = [C.POINTER(abi.CRspectrum), C.c_int, C.c_double, C.c_double, D]
    L.prepare_ic_kernel_flat_cuda.argtypes = [C.POINTER(abi.CRspectrum), C.c_int, C.c_double, C.c_double,
                                              C.c_double, D]
    L.synch_logfx_table_cuda.argtypes = [C.c_int, D, D]
    zero = np.zeros(nb)
    gp = abi.grid(FIX["p_p"], FIX["dp_p"], zero, 0.0, 0.0)
    ge = abi.grid(FIX["p_e"], FIX["dp_e"], zero, 0.0, 0.0)
    out = np.empty((nbins, nb))
    assert L.prepare_gamma_kernel_flat_cuda(C.byref(gp), nbins, *PRM["egamma"], ref_abi.dptr(out)) == 0, abi.error()
    assert rel_to_max(out, FIX["fga"]) <= 1e-11
    assert L.prepare_neutrino_kernel_flat_cuda(C.byref(gp), nbins, *PRM["enu"], ref_abi.dptr(out)) == 0, abi.error()
    assert rel_to_max(out, FIX["fnu"]) <= 1e-11
    assert L.prepare_ic_kernel_flat_cuda(C.byref(ge), nbins, *PRM["nu_ic"], PRM["z_ic"], ref_abi.dptr(out)) == 0
    assert rel_to_max(out, FIX["fic"]) <= 1e-11
    logx = np.ascontiguousarray(FIX["syn_logx"])
    lf = np.empty_like(logx)
    assert L.synch_logfx_table_cuda(len(logx), ref_abi.dptr(logx), ref_abi.dptr(lf)) == 0, abi.error()
    assert float(np.max(np.abs(10.0 ** (lf - FIX["syn_logfx"]) - 1.0))) <= 1e-13


def _resident_context():
    cfg = config.config1(nb=PRM["nb"])
    fp = native.TracerFP(cfg, path="fused")
    fp.set_state(FIX["crp"], FIX["cre"])
    fp.emission_setup(nfreq=PRM["nfreq"], nu_min_s=PRM["nu_s"][0], nu_max_s=PRM["nu_s"][1],
                      ntheta_pitch=PRM["ntheta"], nlogb=PRM["nlogb"], logb_min=PRM["logb"][0],
                      logb_max=PRM["logb"][1], nbins_ic=PRM["nbins"], nu_min_ic=PRM["nu_ic"][0],
                      nu_max_ic=PRM["nu_ic"][1], nbins_gamma=PRM["nbins"], egamma_min=PRM["egamma"][0],
                      egamma_max=PRM["egamma"][1], nbins_nu=PRM["nbins"], enu_min=PRM["enu"][0],
                      enu_max=PRM["enu"][1])
    bg = np.zeros((8, FIX["crp"].shape[0]))
    bg[0] = FIX["n_gas"]
    bg[2] = FIX["b_field"]
    return fp, bg


@pytest.mark.gpu
def test_resident_emission_matches_reference():
    fp, bg = _resident_context()
    try:
        eps = fp.emission_run(bg, PRM["z_ic"])
        table = fp.emission_table("synch", (PRM["nlogb"], PRM["nfreq"], PRM["nb"]))
        fic = fp.emission_table("ic", (PRM["nbins"], PRM["nb"]))
    finally:
        fp.close()
    assert rel_to_max(table[::PRM["plane_stride"]], FIX["syn_table_planes"]) <= 1e-11
    assert rel_to_max(fic, FIX["fic"]) <= 1e-11
    assert rel_to_max(eps["syn"], FIX["eps_syn"]) <= 1e-11
    assert rel_to_max(eps["ic"], FIX["eps_ic"]) <= 1e-11
    assert rel_to_max(eps["gamma"], FIX["eps_gamma"]) <= 1e-11
    assert rel_to_max(eps["nu"], FIX["eps_nu"]) <= 1e-11


@pytest.mark.gpu
def test_resident_emission_device_pointers_equal_host_call():
    torch = pytest.importorskip("torch")
    fp, bg = _resident_context()
    try:
        host = fp.emission_run(bg, PRM["z_ic"])
        n = bg.shape[1]
        d_bg = torch.from_numpy(bg).cuda()
        outs = {k: torch.empty((n, v.shape[1]), dtype=torch.float64, device="cuda") for k, v in host.items()}
        fp.emission_run_device(d_bg.data_ptr(), PRM["z_ic"], **{k: t.data_ptr() for k, t in outs.items()})
        fp.sync()
        for k, t in outs.items():
            assert np.array_equal(t.cpu().numpy(), host[k]), k
    finally:
        fp.close()


@pytest.mark.gpu
@pytest.mark.parametrize("ntr", [1, 3, 9])
def test_resident_emission_ragged_tracer_counts(ntr):
    """Tracer counts below and across the synchrotron kernel's block of 8
    sorted tracers (1, 3, 9), and a setup with only some kinds: each tracer's
    emissivities equal the same tracer's from the 12-tracer run."""
    full, bg = _resident_context()
    try:
        ref = full.emission_run(bg, PRM["z_ic"])
    finally:
        full.close()
    cfg = config.config1(nb=PRM["nb"])
    fp = native.TracerFP(cfg, path="fused")
    try:
        idx = np.arange(ntr) * 5 % FIX["crp"].shape[0]
        fp.set_state(FIX["crp"][idx], FIX["cre"][idx])
        fp.emission_setup(nfreq=PRM["nfreq"], nu_min_s=PRM["nu_s"][0], nu_max_s=PRM["nu_s"][1],
                          ntheta_pitch=PRM["ntheta"], nlogb=PRM["nlogb"], logb_min=PRM["logb"][0],
                          logb_max=PRM["logb"][1], nbins_gamma=PRM["nbins"], egamma_min=PRM["egamma"][0],
                          egamma_max=PRM["egamma"][1])
        eps = fp.emission_run(np.ascontiguousarray(bg[:, idx]), PRM["z_ic"], kinds=("syn", "gamma"))
    finally:
        fp.close()
    assert set(eps) == {"syn", "gamma"}
    for k in eps:
        assert rel_to_max(eps[k], ref[k][idx]) <= 1e-13, k
