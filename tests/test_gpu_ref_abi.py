"""The reference-compatible C ABI (include/fp_cuda_backend.h) on the GPU,
driven through ctypes exactly as CROMA's snapshot driver calls it
(include/tracer_fp_solve.inc:1341-1463), against the CPU restatement.

Bar: spectra within 1e-10 relative on bins above 1e-12 of each tracer's
peak; the emission and batch-solve entry points within 1e-12."""
import ctypes as C
import os

import numpy as np
import pytest

import pyoracle
from conftest import load_package
from golden_io import rel_err

load_package()
from croma_fp_b200 import config, ref_abi, synth  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def _setup(nb=128, nt=40, dpp="asa", seed=21):
    cfg = config.config1(nb=nb, dpp_mode=dpp)
    o = pyoracle.Oracle(cfg)
    abi = ref_abi.RefAbi(nb)
    assert abi.lib.croma_b200_set_model(cfg.dpp_model_id(), cfg.ttd_tacc_model, cfg.t_acc_direct_gyr,
                                        cfg.eta_dpp_cap) == 0
    w = synth.Workload(cfg, nt, 100, seed=seed)
    gp, ge = o.grid(0), o.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    rng = np.random.default_rng(seed)
    qpi = rng.uniform(0.0, 1e45, crp.shape)
    qepri = rng.uniform(0.0, 1e45, cre.shape)
    dis = (np.arange(nt) % 4 == 1).astype(np.uint8)
    return cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis


def _coeff(bg, ric, m1, p1, mass, dis, nxt=None, alpha=0.0):
    ci = ref_abi.FpCoeffBatchInput()
    ci.ncell = bg.shape[1]
    ci.epmax = 1.0e7
    f = [np.ascontiguousarray(bg[k]) for k in range(8)]
    ci.n_gas, ci.kbt, ci.b_field, ci.divv_gyr = (ref_abi.dptr(x) for x in f[:4])
    ci.l_turb_mpc, ci.dv_imc, ci.cs, ci.beta_pl = (ref_abi.dptr(x) for x in f[4:])
    ci.rad_ic_batch, ci.rad_ic_m1, ci.rad_ic_p1 = ref_abi.dptr(ric), ref_abi.dptr(m1), ref_abi.dptr(p1)
    ci.tracer_mass_msun = ref_abi.dptr(mass)
    ci.disable_adiabatic = ref_abi.u8ptr(dis)
    keep = [f, ric, m1, p1, mass, dis]
    if nxt is not None:
        bgn, ricn = nxt
        g = [np.ascontiguousarray(bgn[k]) for k in range(8)]
        ci.device_interp_background = 1
        ci.interp_alpha = alpha
        ci.n_gas_next, ci.kbt_next, ci.b_field_next, ci.divv_gyr_next = (ref_abi.dptr(x) for x in g[:4])
        ci.l_turb_mpc_next, ci.dv_imc_next, ci.cs_next, ci.beta_pl_next = (ref_abi.dptr(x) for x in g[4:])
        ci.rad_ic_batch_next = ref_abi.dptr(ricn)
        keep += [g, ricn]
    return ci, keep


def _pipeline_input(abi, cgp, cge, ci, nstep, dt, windowed, on0, on1, ws):
    pin = abi.PipelineInput()
    pin.ncell = ci.ncell
    pin.nstep = nstep
    pin.fp_cadence_steps = pin.diff_cadence_steps = pin.adv_cadence_steps = 1
    pin.use_windowed_reacc = int(windowed)
    pin.on_start_step, pin.on_end_step = on0, on1
    pin.dt = dt
    pin.epmax = 1.0e7
    pin.psi_value = 0.5
    pin.mach_limit_value = 0.5
    pin.transport_mode = 1
    pin.crp_grid = C.pointer(cgp)
    pin.cre_grid = C.pointer(cge)
    pin.coeff_in = C.pointer(ci)
    pin.workspace = ws
    return pin


@pytest.mark.parametrize("windowed", [False, True])
def test_run_tracer_pipeline_matches_oracle(windowed):
    cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis = _setup()
    nt = crp.shape[0]
    bg = w.background(7)
    row, m1, p1 = o.ic_row(0.6)
    ric = np.ascontiguousarray(np.repeat(row[:, None], nt, axis=1))
    m1s, p1s = np.full(nt, m1), np.full(nt, p1)
    nstep, dt = 9, 2.0e-4
    on0, on1 = (2, 6) if windowed else (0, nstep)
    o_crp, o_cre = crp.copy(), cre.copy()
    o.evolve_segment(nstep, dt, windowed, on0, on1, bg, ric, m1s, p1s, qpi, qepri, o_crp, o_cre,
                     mass=w.mass, dis=dis)
    cgp, cge = abi.grid(*gp), abi.grid(*ge)
    ws = abi.lib.cuda_pipeline_workspace_create()
    assert ws
    try:
        ci, keep = _coeff(bg, ric, m1s, p1s, w.mass, dis)
        pin = _pipeline_input(abi, cgp, cge, ci, nstep, dt, windowed, on0, on1, ws)
        pin.crp_init, pin.cre_init = ref_abi.dptr(crp), ref_abi.dptr(cre)
        pin.qpi_batch, pin.qepri_batch = ref_abi.dptr(qpi), ref_abi.dptr(qepri)
        g_crp, g_cre = np.empty_like(crp), np.empty_like(cre)
        times = ref_abi.FpCudaPipelineTimes()
        rc = abi.lib.run_tracer_pipeline(C.byref(pin), None, ref_abi.dptr(g_crp), ref_abi.dptr(g_cre),
                                         None, None, None, C.byref(times))
        assert rc == 0, abi.error()
        assert rel_err(g_crp, o_crp) <= RTOL
        assert rel_err(g_cre, o_cre) <= RTOL
        assert times.total_ms > 0.0
    finally:
        abi.lib.cuda_pipeline_workspace_destroy(ws)


def test_rank_state_gather_scatter_and_device_interp():
    cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis = _setup(nt=64, dpp="ttd", seed=5)
    nt = crp.shape[0]
    bg0, bg1 = w.background(3), w.background(4)
    r0, m10, p10 = o.ic_row(0.8)
    r1, m11, p11 = o.ic_row(0.78)
    alpha = 0.3125
    bgi = bg0 + alpha * (bg1 - bg0)
    rowi = r0 + alpha * (r1 - r0)
    ric0 = np.ascontiguousarray(np.repeat(r0[:, None], nt, axis=1))
    ric1 = np.ascontiguousarray(np.repeat(r1[:, None], nt, axis=1))
    rici = np.ascontiguousarray(np.repeat(rowi[:, None], nt, axis=1))
    members = np.ascontiguousarray(np.arange(nt)[::-1][: nt // 2].astype(np.int32))
    n = members.size
    nstep, dt = 7, 5.0e-4
    o_crp, o_cre = crp[members].copy(), cre[members].copy()
    o.evolve_segment(nstep, dt, False, 0, nstep, np.ascontiguousarray(bgi[:, members]),
                     np.ascontiguousarray(rici[:, members]), np.full(n, m10), np.full(n, p10),
                     np.ascontiguousarray(qpi[members]), np.ascontiguousarray(qepri[members]),
                     o_crp, o_cre, mass=w.mass[members], dis=dis[members])
    cgp, cge = abi.grid(*gp), abi.grid(*ge)
    ws = abi.lib.cuda_pipeline_workspace_create()
    try:
        t = C.c_double()
        assert abi.lib.cuda_rank_state_upload(ws, nt, ref_abi.dptr(qpi), ref_abi.dptr(qepri),
                                              ref_abi.dptr(crp), ref_abi.dptr(cre), C.byref(t)) == 0
        sub = lambda a: np.ascontiguousarray(a[:, members])
        ci, keep = _coeff(sub(bg0), sub(ric0), np.full(n, m10), np.full(n, p10), w.mass[members].copy(),
                          dis[members].copy(), nxt=(sub(bg1), sub(ric1)), alpha=alpha)
        pin = _pipeline_input(abi, cgp, cge, ci, nstep, dt, False, 0, nstep, ws)
        pin.rank_state_indices = ref_abi.iptr(members)
        pin.gather_rank_state = 1
        pin.scatter_rank_state = 1
        rc = abi.lib.run_tracer_pipeline(C.byref(pin), None, None, None, None, None, None, None)
        assert rc == 0, abi.error()
        d_crp, d_cre = np.empty_like(crp), np.empty_like(cre)
        assert abi.lib.cuda_rank_state_download(ws, nt, ref_abi.dptr(d_crp), ref_abi.dptr(d_cre),
                                                C.byref(t)) == 0
        assert rel_err(d_crp[members], o_crp) <= RTOL
        assert rel_err(d_cre[members], o_cre) <= RTOL
        untouched = np.setdiff1d(np.arange(nt), members)
        assert np.array_equal(d_crp[untouched], crp[untouched])
        assert np.array_equal(d_cre[untouched], cre[untouched])
    finally:
        abi.lib.cuda_pipeline_workspace_destroy(ws)


def _thomas_np(a, b, c, x):
    """fp_thomas_solve_ws (src/fp_shared_core.c:226-257) over rows of a batch."""
    n = a.shape[1]
    x = x.copy()
    cp = np.zeros_like(a)
    cp[:, 0] = -c[:, 0] / b[:, 0]
    x[:, 0] /= b[:, 0]
    for i in range(1, n):
        den = b[:, i] + a[:, i] * cp[:, i - 1]
        cp[:, i] = 0.0 if i == n - 1 else -c[:, i] / den
        x[:, i] = (x[:, i] + a[:, i] * x[:, i - 1]) / den
    for i in range(n - 2, -1, -1):
        x[:, i] -= cp[:, i] * x[:, i + 1]
    return x


def test_solve_cc_cuda_batch_matches_thomas():
    cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis = _setup(nt=32)
    row, m1, p1 = o.ic_row(0.4)
    ric = np.repeat(row[:, None], 32, axis=1)
    ccp_on, cce_on, _, _ = o.cc_coeffs(3e-4, w.background(2), ric, np.full(32, m1), np.full(32, p1), mass=w.mass)
    a, b, c = (np.ascontiguousarray(cce_on[k]) for k in range(3))
    src = np.ascontiguousarray(qepri)
    x0 = np.ascontiguousarray(cre)
    dt = 3e-4
    ref = _thomas_np(a, b, c, dt * src + x0)
    inp = ref_abi.FpChangCooperSolveBatchInput(32, 128, dt, ref_abi.dptr(a), ref_abi.dptr(b), ref_abi.dptr(c),
                                               ref_abi.dptr(src))
    out = np.empty_like(x0)
    ms = C.c_double()
    pcr = C.c_int(7)
    assert abi.lib.solve_cc_cuda_batch(C.byref(inp), ref_abi.dptr(x0), ref_abi.dptr(out), C.byref(ms),
                                       C.byref(pcr)) == 0, abi.error()
    assert pcr.value == 0
    assert rel_err(out, ref) <= 1e-12


def test_hadronic_and_synch_emission_match_restatement():
    cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis = _setup(nt=24)
    nb, nt = 128, 24
    rng = np.random.default_rng(2)
    nbins = 16
    kern = np.ascontiguousarray(rng.uniform(0.0, 1e-30, (nbins, nb)))
    beta_p = o.beta_p()
    n_gas = w.background(0)[0].copy()
    e_min, e_max = -2.0, 6.0
    # Q_one (src/EMISSION.c:297-308) and the energy grid of fp_shared_core.c:2178-2188
    d = (e_max - e_min) / nbins
    a = e_min - d
    E = []
    for _ in range(nbins):
        a += d
        E.append(10.0 ** a)
    f = beta_p[None, None, :] * crp[:, None, :] * kern[None, :, :]
    q = 0.5 * np.sum((f[:, :, :-1] + f[:, :, 1:]) * gp[1][None, None, 1:], axis=2)
    ref = np.array(E)[None, :] * q * n_gas[:, None]
    inp = ref_abi.FpHadronicEmissionBatchInput(nt, nbins, 0.0, e_min, e_max, ref_abi.dptr(n_gas),
                                               ref_abi.dptr(crp), ref_abi.dptr(beta_p), ref_abi.dptr(kern))
    cg = abi.grid(*gp)
    out = np.empty((nt, nbins))
    ms = C.c_double()
    for fn in (abi.lib.prepare_gamma_emission_cuda_batch, abi.lib.prepare_neutrino_emission_cuda_batch):
        assert fn(C.byref(inp), C.byref(cg), ref_abi.dptr(out), C.byref(ms)) == 0, abi.error()
        assert rel_err(out, ref, 1e-30) <= 1e-12

    # synchrotron, pitch-kernel-table branch (fp_shared_core.c:2070-2112)
    nfreq, nlogb = 8, 32
    table = np.ascontiguousarray(rng.uniform(1e-3, 1.0, (nlogb, nfreq, nb)))
    table[3, :, 10:20] = 0.0
    b_dyn = np.ascontiguousarray(w.background(0)[2])
    logb = np.ascontiguousarray(np.log10(b_dyn))
    logb_min, inv_dlogb = -9.0, nlogb / 5.0
    ref = np.zeros((nt, nfreq))
    for i in range(nt):
        A = np.sqrt(3.0) * (4.8e-10 ** 3) * b_dyn[i] / (2.0 * 9.11e-28 * 2.999e10 * 2.999e10) / (4.0 * np.pi)
        u = (logb[i] - logb_min) * inv_dlogb
        ib = int(np.clip(np.floor(u), 0, nlogb - 2))
        t = float(np.clip(u - ib, 0.0, 1.0))
        for nf in range(nfreq):
            s = 0.0
            je = 2
            while je < nb - 1 and cre[i, je + 1] > 0.0:
                k0, k1 = table[ib, nf, je], table[ib + 1, nf, je]
                if t <= 0.0:
                    K = k0
                elif t >= 1.0:
                    K = k1
                elif k0 > 0 and k1 > 0:
                    K = np.exp((1 - t) * np.log(k0) + t * np.log(k1))
                else:
                    K = (1 - t) * k0 + t * k1
                s += cre[i, je] * K * ge[1][je]
                je += 1
            ref[i, nf] = A * s
    sin = ref_abi.FpSynchEmissionBatchInput()
    sin.ncell, sin.nfreq, sin.nlogb = nt, nfreq, nlogb
    sin.logb_min, sin.inv_dlogb = logb_min, inv_dlogb
    sin.pitch_kernel_table = ref_abi.dptr(table)
    sin.b_dyn, sin.logb, sin.cre_batch = ref_abi.dptr(b_dyn), ref_abi.dptr(logb), ref_abi.dptr(cre)
    out = np.empty((nt, nfreq))
    assert abi.lib.prepare_synch_emission_cuda_batch(C.byref(sin), C.byref(abi.grid(*ge)), ref_abi.dptr(out),
                                                     C.byref(ms)) == 0, abi.error()
    assert rel_err(out, ref, 1e-30) <= 1e-12


def test_device_binding_entry_points():
    abi = ref_abi.RefAbi(128)
    assert abi.lib.cuda_pipeline_is_available() == 1
    dev = C.c_int(-1)
    assert abi.lib.cuda_bind_local_rank(0, C.byref(dev)) == 0 and dev.value == 0
    cnt, cur = C.c_int(), C.c_int()
    assert abi.lib.cuda_get_binding_state(C.byref(cnt), C.byref(cur)) == 0
    assert cnt.value >= 1 and cur.value == 0
    buf = C.create_string_buffer(64)
    assert abi.lib.cuda_get_current_device_id(buf, 64) == 0 and len(buf.value) > 4
    assert abi.lib.fp_cuda_tridiag_uses_pcr(128) == 0
    assert b"Thomas" in abi.lib.fp_cuda_tridiag_solver_name(128)


def test_solve_cc_cuda_batch_pcr_when_requested(monkeypatch):
    """CROMA_CUDA_TRIDIAG=pcr (src/fp_cuda_solver.cu:41-72): the batch solve
    runs parallel cyclic reduction and reports it; same result as Thomas."""
    cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis = _setup(nt=16)
    row, m1, p1 = o.ic_row(0.4)
    ric = np.repeat(row[:, None], 16, axis=1)
    _, cce_on, _, _ = o.cc_coeffs(3e-4, w.background(2), ric, np.full(16, m1), np.full(16, p1), mass=w.mass)
    a, b, c = (np.ascontiguousarray(cce_on[k]) for k in range(3))
    src, x0, dt = np.ascontiguousarray(qepri), np.ascontiguousarray(cre), 3e-4
    ref = _thomas_np(a, b, c, dt * src + x0)
    inp = ref_abi.FpChangCooperSolveBatchInput(16, 128, dt, ref_abi.dptr(a), ref_abi.dptr(b), ref_abi.dptr(c),
                                               ref_abi.dptr(src))
    monkeypatch.setenv("CROMA_CUDA_TRIDIAG", "pcr")
    assert abi.lib.fp_cuda_tridiag_uses_pcr(128) == 1
    assert abi.lib.fp_cuda_tridiag_uses_pcr(100) == -1
    out, ms, pcr = np.empty_like(x0), C.c_double(), C.c_int(7)
    assert abi.lib.solve_cc_cuda_batch(C.byref(inp), ref_abi.dptr(x0), ref_abi.dptr(out), C.byref(ms),
                                       C.byref(pcr)) == 0, abi.error()
    assert pcr.value == 1
    assert rel_err(out, ref) <= 1e-12
    monkeypatch.setenv("CROMA_CUDA_TRIDIAG", "thomas")
    assert abi.lib.fp_cuda_tridiag_uses_pcr(128) == 0


CALLER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                      "abi_caller_np128")


@pytest.mark.skipif(not os.path.exists(CALLER), reason="C caller not built (needs the reference's headers)")
def test_c_caller_compiled_against_reference_header():
    """oracle/abi_caller.c, compiled against the reference's own
    fp_cuda_backend.h / fp_shared_core.h / params.h and linked to
    libcroma_b200_np128.so, runs cuda_rank_state_upload -> run_tracer_pipeline
    (gather and scatter through the rank state) -> cuda_rank_state_download;
    its spectra match the oracle's segment within 1e-10."""
    import subprocess
    import tempfile
    cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis = _setup(nt=48, seed=33)
    nt = crp.shape[0]
    bg = w.background(9)
    row, m1, p1 = o.ic_row(0.55)
    ric = np.ascontiguousarray(np.repeat(row[:, None], nt, axis=1))
    m1s, p1s = np.full(nt, m1), np.full(nt, p1)
    nstep, dt, windowed, on0, on1 = 7, 3.0e-4, 1, 1, 5
    o_crp, o_cre = crp.copy(), cre.copy()
    o.evolve_segment(nstep, dt, windowed, on0, on1, bg, ric, m1s, p1s, qpi, qepri, o_crp, o_cre,
                     mass=w.mass, dis=dis)
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(np.array([nt, nstep, windowed, on0, on1, cfg.dpp_model_id(), cfg.ttd_tacc_model],
                             np.int32).tobytes())
            f.write(np.array([dt, cfg.t_acc_direct_gyr, cfg.eta_dpp_cap]).tobytes())
            for g in (gp, ge):
                f.write(np.concatenate([g[0], g[1], g[2], [g[3], g[4]]]).astype(np.float64).tobytes())
            for a in (bg, ric, m1s, p1s, w.mass):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
            f.write(np.ascontiguousarray(dis, np.uint8).tobytes())
            for a in (crp, cre, qpi, qepri):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
        r = subprocess.run([CALLER, fin, fout], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        out = np.fromfile(fout, np.float64)
    g_crp, g_cre = out[:nt * 128].reshape(nt, 128), out[nt * 128:].reshape(nt, 128)
    assert rel_err(g_crp, o_crp) <= RTOL
    assert rel_err(g_cre, o_cre) <= RTOL


def test_run_tracer_pipeline_with_pcr_requested(monkeypatch):
    """CROMA_CUDA_TRIDIAG=pcr in the pipeline: the steps kernel runs warp PCR,
    FpCudaPipelineTimes reports it for both species, and the spectra still
    match the oracle's segment within 1e-10."""
    monkeypatch.setenv("CROMA_CUDA_TRIDIAG", "pcr")
    cfg, o, abi, w, gp, ge, crp, cre, qpi, qepri, dis = _setup(nt=24, seed=41)
    nt = crp.shape[0]
    bg = w.background(11)
    row, m1, p1 = o.ic_row(0.45)
    ric = np.ascontiguousarray(np.repeat(row[:, None], nt, axis=1))
    m1s, p1s = np.full(nt, m1), np.full(nt, p1)
    nstep, dt = 6, 2.5e-4
    o_crp, o_cre = crp.copy(), cre.copy()
    o.evolve_segment(nstep, dt, False, 0, nstep, bg, ric, m1s, p1s, qpi, qepri, o_crp, o_cre, mass=w.mass, dis=dis)
    cgp, cge = abi.grid(*gp), abi.grid(*ge)
    ws = abi.lib.cuda_pipeline_workspace_create()
    assert ws
    try:
        ci, keep = _coeff(bg, ric, m1s, p1s, w.mass, dis)
        pin = _pipeline_input(abi, cgp, cge, ci, nstep, dt, False, 0, nstep, ws)
        pin.crp_init, pin.cre_init = ref_abi.dptr(crp), ref_abi.dptr(cre)
        pin.qpi_batch, pin.qepri_batch = ref_abi.dptr(qpi), ref_abi.dptr(qepri)
        g_crp, g_cre = np.empty_like(crp), np.empty_like(cre)
        times = ref_abi.FpCudaPipelineTimes()
        rc = abi.lib.run_tracer_pipeline(C.byref(pin), None, ref_abi.dptr(g_crp), ref_abi.dptr(g_cre),
                                         None, None, None, C.byref(times))
        assert rc == 0, abi.error()
        assert times.used_pcr_proton == 1 and times.used_pcr_electron == 1
        assert rel_err(g_crp, o_crp) <= RTOL
        assert rel_err(g_cre, o_cre) <= RTOL
    finally:
        abi.lib.cuda_pipeline_workspace_destroy(ws)
