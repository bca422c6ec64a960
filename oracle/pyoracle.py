"""ctypes front-ends for the two checkers.

* ``Oracle``       -- the CPU restatement (oracle/croma_oracle.c,
                      built as oracle/_build/liboracle.so).
* ``ReferenceCPU`` -- the reference's own CPU sources compiled as-is with
                      oracle/ref_driver.c (oracle/_ref/libcroma_ref_np<N>.so);
                      present only where the reference tree was available at
                      build time.

Test infrastructure: only tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py import this module, and only to check or time
the reference algorithm.  Both expose the same methods with numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_U8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_i = C.c_int
_d = C.c_double


class _Params(C.Structure):
    _fields_ = [("nb", _i), ("pmin", _d), ("pmax", _d), ("pemin", _d), ("pemax", _d),
                ("dpp_model", _i), ("ttd_tacc_model", _i), ("t_acc_direct_gyr", _d),
                ("mach_limit", _d), ("psi", _d), ("eta_dpp_cap", _d), ("nsub_safety", _d),
                ("nsub_max", _i), ("coeff_interp_min_steps", _i),
                ("coeff_interp_max_segments", _i), ("reacc_window_mode", _i), ("f_eddy", _d),
                ("t_off_gyr", _d), ("t_acc_off_gyr", _d)]


class _RefConfig(C.Structure):
    _fields_ = [("pmin", _d), ("pmax", _d), ("pemin", _d), ("pemax", _d), ("dpp_model", _i),
                ("ttd_tacc_model", _i), ("t_acc_direct_gyr", _d), ("mach_limit", _d),
                ("psi", _d), ("eta_dpp_cap", _d), ("nsub_safety", _d), ("nsub_max", _i),
                ("coeff_interp_min_steps", _i), ("coeff_interp_max_segments", _i),
                ("reacc_window_mode", _i), ("f_eddy", _d), ("t_off_gyr", _d),
                ("t_acc_off_gyr", _d), ("nthreads", _i)]


class _DsaParams(C.Structure):
    _fields_ = [("eta_model_initial", _i), ("eta_model_reacc", _i), ("chi_p", _d), ("chi_e", _d),
                ("k_ep", _d), ("pmax_p_mc", _d), ("pmax_e_mc", _d), ("min_mach", _d),
                ("gamma_gas", _d), ("xcr_pmin_pmc", _d), ("reacc_eta_cap", _d), ("mu_mol", _d),
                ("pmin_dsa_p_log10", _d), ("pmin_dsa_e_log10", _d), ("inject_species", _i)]


SHOCK_FIELDS = ("mach", "prestemp", "presden", "pre_density_cgs", "upstream_speed_cgs",
                "shock_side_code", "dsa_trigger", "dsa_mach", "dsa_pre_density", "dsa_flux_cgs")


class _ShockFields(C.Structure):
    _fields_ = [(n, _vp) for n in SHOCK_FIELDS] + [("has_dsa", _i)]


def _dsa_structs(params, shocks):
    """ctypes structs for DSA parameters (an object with the _DsaParams
    field names) and shock fields (dict of [ntracer] arrays, missing = NULL,
    plus 'has_dsa'); the arrays are kept alive in the returned tuple."""
    prm = _DsaParams()
    for name, _ in _DsaParams._fields_:
        setattr(prm, name, getattr(params, name))
    keep = {}
    sh = _ShockFields()
    for n in SHOCK_FIELDS:
        a = shocks.get(n)
        if a is not None:
            keep[n] = np.ascontiguousarray(a, dtype=np.float64)
            setattr(sh, n, keep[n].ctypes.data)
    sh.has_dsa = int(shocks.get("has_dsa", 0))
    return prm, sh, keep


def _fill(struct, cfg, extra=None):
    s = struct()
    for name, _ in struct._fields_:
        if name == "dpp_model":
            s.dpp_model = cfg.dpp_model_id()
        elif extra and name in extra:
            setattr(s, name, extra[name])
        elif hasattr(cfg, name):
            setattr(s, name, getattr(cfg, name))
    return s


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _as_d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class _Common:
    nb: int

    def grid(self, species: int):
        """(p, dp, E, pm1, pp1) for species 0 = proton, 1 = electron."""
        out = np.empty(3 * self.nb + 2)
        self._get_grid(species, out)
        n = self.nb
        return out[:n].copy(), out[n:2 * n].copy(), out[2 * n:3 * n].copy(), out[3 * n], out[3 * n + 1]

    def ic_row(self, z: float):
        row = np.empty(self.nb)
        m1, p1 = _d(), _d()
        self._ic_row(z, row, m1, p1)
        return row, m1.value, p1.value

    def pp_cache(self):
        s = np.empty(self.nb); g = np.empty(self.nb); j = _i()
        self._pp_cache(s, g, j)
        return s, g, j.value

    def secondary_kernel(self):
        f = np.empty(self.nb * self.nb); m = np.empty(self.nb, dtype=np.int32)
        self._sec(f, m)
        return f.reshape(self.nb, self.nb), m

    def nsub(self, dt_snap: float, bg: np.ndarray, rad_ic_row: np.ndarray):
        n = bg.shape[1]
        nsub = np.empty(n, np.int32); tgt = np.empty(n, np.int32); non = np.empty(n, np.int32)
        cap = np.zeros(n, np.uint8)
        err = self._nsub(n, dt_snap, _as_d(bg), _as_d(rad_ic_row), nsub, tgt, non, cap)
        if err != 0:
            raise RuntimeError(f"nsub failed: {err}")
        return nsub, tgt, non, cap

    def dsa_inject(self, params, shocks, mass, density_unit, dt_gyr, mode, reacc_mode, crp, cre,
                   qpi=None, qepri=None, dis=None):
        """tracer_fp_apply_dsa_tracer_injection_snapshot on cell-major arrays
        (modified in place).  Returns the number of tracers injected."""
        prm, sh, keep = _dsa_structs(params, shocks)
        n = crp.shape[0]
        nin = _i()
        rc = self._dsa(C.byref(prm), C.byref(sh), n, _ptr(_as_d(mass)), float(density_unit),
                       float(dt_gyr), int(mode), int(reacc_mode), _ptr(crp), _ptr(cre), _ptr(qpi),
                       _ptr(qepri), _ptr(dis), C.byref(nin))
        if rc != 0:
            raise RuntimeError(f"dsa_inject failed: {rc}")
        return nin.value

    def buckets(self, nsub: np.ndarray, non: np.ndarray):
        n = nsub.size
        bid = np.empty(n, np.int32); idx = np.empty(n, np.int32)
        steps = np.empty(n, np.int32); ons = np.empty(n, np.int32)
        offs = np.empty(n, np.int32); cnts = np.empty(n, np.int32); nb = _i()
        self._buckets(n, np.ascontiguousarray(nsub, np.int32), np.ascontiguousarray(non, np.int32),
                      bid, idx, steps, ons, offs, cnts, C.byref(nb))
        k = nb.value
        return dict(bucket_ids=bid, indices=idx, steps=steps[:k].copy(), onsteps=ons[:k].copy(),
                    offsets=offs[:k].copy(), counts=cnts[:k].copy(), nbuckets=k)


class Oracle(_Common):
    """The CPU restatement (runtime bin count)."""

    def __init__(self, cfg, threads: int = 0):
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle restated`")
        L = C.CDLL(path)
        self.lib = L
        L.or_create.restype = _vp
        L.or_create.argtypes = [C.POINTER(_Params)]
        L.or_destroy.argtypes = [_vp]
        L.or_get_grid.argtypes = [_vp, _i, _D]
        L.or_ic_row.argtypes = [_vp, _d, _D, C.POINTER(_d), C.POINTER(_d)]
        L.or_get_pp_cache.argtypes = [_vp, _D, _D, C.POINTER(_i)]
        L.or_get_secondary_kernel.argtypes = [_vp, _D, _I]
        L.or_get_beta_p.argtypes = [_vp, _D]
        L.or_nsub.argtypes = [_vp, _i, _d, _D, _D, _I, _I, _I, _U8]
        L.or_buckets.argtypes = [_i, _I, _I, _I, _I, _I, _I, _I, _I, C.POINTER(_i)]
        L.or_coeff_segments.argtypes = [_vp, _i, _i]
        L.or_cc_coeffs.argtypes = [_vp, _i, _d, _D, _D, _D, _D, _vp, _vp, _vp, _vp, _D, _D, _D, _D]
        L.or_evolve_segment.argtypes = [_vp, _i, _i, _d, _i, _i, _i, _D, _D, _D, _D, _D, _D,
                                        _vp, _vp, _D, _D]
        L.or_snapshot.argtypes = [_vp, _i, _D, _D, _d, _d, _i, _d, _d, _D, _D, _vp, _vp, _D, _D,
                                  _I, _I, _I, C.POINTER(_i)]
        L.or_snapshot_with_ic.argtypes = [_vp, _i, _D, _D, _D, _D, _i, _d, _d, _D, _D, _vp, _vp,
                                          _D, _D, _I, _I, _I, C.POINTER(_i)]
        L.or_set_threads.argtypes = [_i]
        L.or_dsa_inject.argtypes = [_vp, _i, _vp, _vp, _vp, _vp, _vp, _i, _vp, _d, _d, _i, _i,
                                    _vp, _vp, _vp, _vp, _vp, _vp]
        self.cfg = cfg
        self.nb = cfg.nb
        p = _fill(_Params, cfg)
        self.ctx = L.or_create(C.byref(p))
        if not self.ctx:
            raise RuntimeError("or_create failed")
        if threads:
            L.or_set_threads(threads)

    def __del__(self):
        try:
            self.lib.or_destroy(self.ctx)
        except Exception:
            pass

    def _get_grid(self, s, out): return self.lib.or_get_grid(self.ctx, s, out)
    def _ic_row(self, z, row, m1, p1): return self.lib.or_ic_row(self.ctx, z, row, C.byref(m1), C.byref(p1))
    def _pp_cache(self, s, g, j): return self.lib.or_get_pp_cache(self.ctx, s, g, C.byref(j))
    def _sec(self, f, m): return self.lib.or_get_secondary_kernel(self.ctx, f, m)
    def _nsub(self, *a): return self.lib.or_nsub(self.ctx, *a)
    def _buckets(self, *a): return self.lib.or_buckets(*a)

    def _dsa(self, prm, sh, n, mass, dunit, dt, mode, reacc, crp, cre, qpi, qepri, dis, nin):
        gp, ge = self.grid(0), self.grid(1)
        self._dsa_grids = (np.ascontiguousarray(gp[0]), np.ascontiguousarray(gp[1]),
                           np.ascontiguousarray(ge[0]), np.ascontiguousarray(ge[1]))
        g = [a.ctypes.data for a in self._dsa_grids]
        return self.lib.or_dsa_inject(prm, self.nb, *g, sh, n, mass, dunit, dt, mode, reacc, crp, cre,
                                      qpi, qepri, dis, nin)

    def beta_p(self):
        out = np.empty(self.nb)
        self.lib.or_get_beta_p(self.ctx, out)
        return out

    def coeff_segments(self, nsub: int, allow_interp: bool) -> int:
        return self.lib.or_coeff_segments(self.ctx, int(nsub), int(allow_interp))

    def cc_coeffs(self, dt, bg, rad_ic, rad_ic_m1, rad_ic_p1, mass=None, dis=None, crp=None, cre=None):
        n = bg.shape[1]; nb = self.nb
        outs = [np.empty(3 * n * nb) for _ in range(4)]
        err = self.lib.or_cc_coeffs(self.ctx, n, dt, _as_d(bg), _as_d(rad_ic), _as_d(rad_ic_m1),
                                    _as_d(rad_ic_p1), _ptr(_as_d(mass)),
                                    _ptr(None if dis is None else np.ascontiguousarray(dis, np.uint8)),
                                    _ptr(_as_d(crp)), _ptr(_as_d(cre)), *outs)
        if err != 0:
            raise RuntimeError("cc_coeffs failed")
        return [o.reshape(3, n, nb) for o in outs]

    def evolve_segment(self, nstep, dt, windowed, on_start, on_end, bg, rad_ic, rad_ic_m1,
                       rad_ic_p1, qpi, qepri, crp, cre, mass=None, dis=None):
        n = bg.shape[1]
        err = self.lib.or_evolve_segment(self.ctx, n, nstep, dt, int(windowed), on_start, on_end,
                                         _as_d(bg), _as_d(rad_ic), _as_d(rad_ic_m1), _as_d(rad_ic_p1),
                                         _as_d(qpi), _as_d(qepri), _ptr(_as_d(mass)),
                                         _ptr(None if dis is None else np.ascontiguousarray(dis, np.uint8)),
                                         crp, cre)
        if err != 0:
            raise RuntimeError("evolve_segment failed")

    def snapshot(self, bg_curr, bg_next, z_curr, z_next, allow, dt, elapsed, qpi, qepri, crp, cre,
                 mass=None, dis=None, ic=None):
        """Advance crp/cre (cell-major, in place) through one snapshot.
        ic = (ic_curr, ic_next) rows of nb+2 values to skip the IC integrals."""
        n = bg_curr.shape[1]
        nsub = np.empty(n, np.int32); non = np.empty(n, np.int32); bid = np.empty(n, np.int32)
        nbk = _i()
        dptr = _ptr(None if dis is None else np.ascontiguousarray(dis, np.uint8))
        if ic is None:
            err = self.lib.or_snapshot(self.ctx, n, _as_d(bg_curr), _as_d(bg_next), z_curr, z_next,
                                       int(allow), dt, elapsed, _as_d(qpi), _as_d(qepri),
                                       _ptr(_as_d(mass)), dptr, crp, cre, nsub, non, bid, C.byref(nbk))
        else:
            err = self.lib.or_snapshot_with_ic(self.ctx, n, _as_d(bg_curr), _as_d(bg_next),
                                               _as_d(ic[0]), _as_d(ic[1]), int(allow), dt, elapsed,
                                               _as_d(qpi), _as_d(qepri), _ptr(_as_d(mass)), dptr,
                                               crp, cre, nsub, non, bid, C.byref(nbk))
        if err != 0:
            raise RuntimeError(f"oracle snapshot failed: {err}")
        return nsub, non, bid, nbk.value


def synch_fx(logx, xmin, logx_tab, logfx_tab, fx_tab):
    """F(x) of the log-tabulated synchrotron kernel at each logx, as
    SYN_emissivity_from_arrays looks it up (src/Synchrotron.c:81-97)."""
    nx = len(logx_tab)
    inv_dlogx = 1.0 / (logx_tab[1] - logx_tab[0]) if nx > 1 else 0.0
    logx = np.asarray(logx, dtype=np.float64)
    out = np.zeros_like(logx)
    ok = logx <= logx_tab[nx - 1]
    ix = np.floor((logx - xmin) * inv_dlogx)
    last = ok & (ix >= nx - 1)
    out[last] = fx_tab[nx - 1]
    mid = ok & (ix >= 0) & (ix < nx - 1)
    i = ix[mid].astype(np.int64)
    frac = (logx[mid] - logx_tab[i]) * inv_dlogx
    out[mid] = 10.0 ** (logfx_tab[i] + frac * (logfx_tab[i + 1] - logfx_tab[i]))
    return out


def synch_pitch_table(logy, w, logb_min, inv_dlogb, nlogb, xmin, logx_tab, logfx_tab, fx_tab):
    """prepare_synch_pitch_kernel_table (src/fp_shared_core.c:2008-2052):
    [nlogb][nfreq][npe] = sum_k F(logy[nf][je][k] - logb) w_k."""
    nfreq, nb, _ = logy.shape
    out = np.empty((nlogb, nfreq, nb))
    for ib in range(nlogb):
        logb = logb_min + ib / inv_dlogb
        out[ib] = np.sum(synch_fx(logy - logb, xmin, logx_tab, logfx_tab, fx_tab) * w[None, None, :], axis=2)
    return out


def synch_emission_theta(cre, dp, b_dyn, logb, logy, w, xmin, logx_tab, logfx_tab, fx_tab):
    """prepare_synch_emission_cell_major without a pitch table
    (src/fp_shared_core.c:2113-2120 -> SYN_emissivity_from_arrays,
    src/Synchrotron.c:62-103): eps[cell][nf] = A B-dependent prefactor times
    sum over je = 2 .. (first je with N[je+1] <= 0) of N int_th dp."""
    ncell, nb = cre.shape
    nfreq = logy.shape[0]
    out = np.empty((ncell, nfreq))
    for i in range(ncell):
        A = np.sqrt(3.0) * (4.8e-10 ** 3.0) * b_dyn[i] / (2.0 * 9.11e-28 * 2.999e10 * 2.999e10) \
            / (4.0 * np.pi)
        stop = 2
        while stop < nb - 1 and cre[i, stop + 1] > 0.0:
            stop += 1
        for nf in range(nfreq):
            s = 0.0
            for je in range(2, stop):
                th = float(np.sum(synch_fx(logy[nf, je] - logb[i], xmin, logx_tab, logfx_tab, fx_tab) * w))
                s += cre[i, je] * th * dp[je]
            out[i, nf] = A * s
    return out


_BG_ARGS = ("temp_K", "density", "bx", "by", "bz", "div_v", "curl_v_prev", "curl_v", "curl_v_next", "l_turb_cm")


def background(raw: dict, params: dict) -> np.ndarray:
    """or_background (oracle/croma_oracle_background.c): the [8][n]
    background block from one snapshot's raw fields (the keys of
    CromaB200RawSnapshot) and the run parameters (CromaB200BackgroundParams)."""
    L = C.CDLL(os.path.join(HERE, "_build", "liboracle.so"))
    arrs = [None if raw.get(k) is None else np.ascontiguousarray(raw[k], dtype=np.float64) for k in _BG_ARGS]
    n = arrs[0].shape[0]
    bg = np.empty((8, n))
    L.or_background.restype = _i
    L.or_background.argtypes = [_i] + [_vp] * 10 + [_d] * 5 + [_i, _i, _i] + [_d] * 4 + [_vp]
    rc = L.or_background(n, *[None if a is None else a.ctypes.data for a in arrs], raw["c_dens"], raw["c_mag"],
                         raw["z_prev"], raw["z_curr"], raw["z_next"], int(raw["apply_temp_floor"]),
                         int(raw["allow_curl_interp"]), int(params["bfield_mode"]), params["mu_mol"],
                         params["eta_B"], params["mach_limit"], params["l_turb_target_kpc"], bg.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"or_background returned {rc}")
    return bg


class _BgCellIn(C.Structure):   # FpBackgroundCellInput, include/fp_shared_core.h:207-224
    _fields_ = [(k, _d) for k in ("density_gcc", "temp_K", "bx_G", "by_G", "bz_G", "divv_gyr", "curl_v_s",
                                 "curl_v_prev_s", "curl_v_next_s", "z_prev", "z_curr", "z_next", "l_turb_cm",
                                 "target_l_turb_cm")] + [("apply_temp_floor", _i), ("allow_curl_interp", _i)]


class _BgCellOut(C.Structure):   # FpBackgroundCellOutput, include/fp_shared_core.h:226-239
    _fields_ = [(k, _d) for k in ("n_gas", "kbt_GeV", "b_sim_G", "b_dyn_G", "b_eff_G", "divv_gyr", "l_turb_mpc",
                                 "dv_imc_cms", "cs_cms", "beta_pl", "curl_v_used_s", "temp_used_K")]


def reference_background(raw: dict, params: dict, nb: int = 128) -> np.ndarray:
    """The reference's own prepare_background_cell (compiled in
    oracle/_ref) per tracer, with the raw scaling and the argument forms of
    tracer_load_hdf5_raw_snapshot_slice and tracer_prepare_background_from_raw
    (src/tracer_fp_background.c:1189-1197, 1206-1263) and the stored fields of
    tracer_store_background_history_slot (:324-342)."""
    L = C.CDLL(os.path.join(HERE, "_ref", f"libcroma_ref_np{nb}.so"))
    _i.in_dll(L, "bfield_mode").value = int(params["bfield_mode"])
    _d.in_dll(L, "mu_mol").value = params["mu_mol"]
    _d.in_dll(L, "eta_B").value = params["eta_B"]
    _d.in_dll(L, "mach_limit").value = params["mach_limit"]
    L.prepare_background_cell.restype = _i
    L.prepare_background_cell.argtypes = [C.POINTER(_BgCellIn), C.POINTER(_BgCellOut)]
    n = len(raw["temp_K"])
    target = params["l_turb_target_kpc"] * 3.0857e21
    bg = np.empty((8, n))
    prev = raw.get("curl_v_prev")
    nxt = raw.get("curl_v_next")
    lt = raw.get("l_turb_cm")
    for i in range(n):
        a = _BgCellIn(density_gcc=raw["density"][i] * raw["c_dens"], temp_K=raw["temp_K"][i],
                      bx_G=raw["bx"][i] * raw["c_mag"], by_G=raw["by"][i] * raw["c_mag"],
                      bz_G=raw["bz"][i] * raw["c_mag"], divv_gyr=1.0 * raw["div_v"][i] * 3.1536e16,
                      curl_v_s=1.0 * raw["curl_v"][i], curl_v_prev_s=1.0 * (prev[i] if prev is not None else 0.0),
                      curl_v_next_s=1.0 * (nxt[i] if nxt is not None else 0.0), z_prev=raw["z_prev"],
                      z_curr=raw["z_curr"], z_next=raw["z_next"], l_turb_cm=(lt[i] if lt is not None else 0.0),
                      target_l_turb_cm=target, apply_temp_floor=int(raw["apply_temp_floor"]),
                      allow_curl_interp=int(raw["allow_curl_interp"]))
        o = _BgCellOut()
        if L.prepare_background_cell(C.byref(a), C.byref(o)) != 0:
            raise RuntimeError(f"prepare_background_cell failed at tracer {i}")
        bg[:, i] = (o.n_gas, o.kbt_GeV, o.b_eff_G, o.divv_gyr, o.l_turb_mpc, o.dv_imc_cms, o.cs_cms, o.beta_pl)
    return bg


def reference_available(nb: int) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libcroma_ref_np{nb}.so"))


class ReferenceCPU(_Common):
    """The reference's own CPU code (compile-time bin count)."""

    _loaded = {}

    def __init__(self, cfg, threads: int = 0):
        path = os.path.join(HERE, "_ref", f"libcroma_ref_np{cfg.nb}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        L = C.CDLL(path)
        self.lib = L
        L.ref_configure.argtypes = [C.POINTER(_RefConfig)]
        L.ref_get_grid.argtypes = [_i, _D]
        L.ref_ic_row.argtypes = [_d, _D, C.POINTER(_d), C.POINTER(_d)]
        L.ref_get_pp_cache.argtypes = [_D, _D, C.POINTER(_i)]
        L.ref_get_secondary_kernel.argtypes = [_D, _I]
        L.ref_get_beta_p.argtypes = [_D]
        L.ref_nsub.argtypes = [_i, _d, _D, _D, _I, _I, _I, _U8]
        L.ref_buckets.argtypes = [_i, _I, _I, _I, _I, _I, _I, _I, _I, C.POINTER(_i)]
        L.ref_coeff_segments.argtypes = [_i, _i]
        L.ref_cc_coeffs.argtypes = [_i, _d, _D, _D, _D, _D, _vp, _vp, _vp, _vp, _D, _D, _D, _D]
        L.ref_evolve_segment.argtypes = [_i, _i, _d, _i, _i, _i, _D, _D, _D, _D, _D, _D, _vp, _vp,
                                         _D, _D]
        L.ref_snapshot.argtypes = [_i, _D, _D, _d, _d, _i, _d, _d, _D, _D, _vp, _vp, _D, _D, _I, _I,
                                   _I, C.POINTER(_i)]
        L.ref_dsa_inject.argtypes = [_vp, _vp, _i, _vp, _d, _d, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]
        L.ref_ic_emission.argtypes = [_i, _i, _d, _d, _d, _D, _D, _D]
        L.ref_synch_pitch_table.argtypes = [_i, _i, _i, _i, _d, _d, _d, _D, _D, _D, _D, _D, _D]
        _s, _l = C.c_char_p, C.c_long
        L.ref_tile_open.argtypes = [_s, _s, _i, _l, _l, _l, _i]
        L.ref_tile_write_cr.argtypes = [_i, _i, _i, _l, _vp, _vp, _vp, _vp, _i, _i]
        L.ref_tile_write_emit.argtypes = [_i, _i, _l, _i, _vp, _vp, _vp, _i]
        L.ref_tile_close.argtypes = [_i]
        L.ref_map_open.argtypes = [_s, _s, _i, _i, _l, _i]
        L.ref_write_cr_map.argtypes = [_i, _i, _i, _i, _vp, _vp, _vp, _vp, _i]
        L.ref_write_emit_map.argtypes = [_i, _i, _i, _i, _vp, _vp, _vp, _i]
        L.ref_map_close.argtypes = [_i]
        L.ref_ckpt_write.argtypes = [_s, _i, _i, _i, _i, _i, _i, _i, _l, _vp, _vp, _vp, _i, _i]
        L.ref_ckpt_read.argtypes = [_s, _i, _i, _i, _i, _i, _i, _l, _vp, _vp, _vp, _i, _i, C.POINTER(_i)]
        L.ref_synch_emission.argtypes = [_i, _i, _i, _i, _i, _d, _d, _d, _D, _D, _D, _D, _D, _vp, _D, _D,
                                         _D, _D]
        L.ref_gamma_kernel_table.argtypes = [_i, _d, _d, _D]
        L.ref_nu_kernel_table.argtypes = [_i, _d, _d, _D]
        L.ref_ic_kernel_table.argtypes = [_i, _d, _d, _d, _D]
        L.ref_hadronic_emission.argtypes = [_i, _i, _i, _d, _d, _D, _D, _D, _D]
        L.ref_synch_run.argtypes = [_i, _d, _d, _i, _i, _d, _d, _i, _vp, _vp] + [_vp] * 9
        self.cfg = cfg
        self.nb = cfg.nb
        self.configure(threads)

    def configure(self, threads: int = 0):
        rc = _fill(_RefConfig, self.cfg, {"nthreads": threads})
        if self.lib.ref_configure(C.byref(rc)) != 0:
            raise RuntimeError("ref_configure failed")

    def _get_grid(self, s, out): return self.lib.ref_get_grid(s, out)
    def _ic_row(self, z, row, m1, p1): return self.lib.ref_ic_row(z, row, C.byref(m1), C.byref(p1))
    def _pp_cache(self, s, g, j): return self.lib.ref_get_pp_cache(s, g, C.byref(j))
    def _sec(self, f, m): return self.lib.ref_get_secondary_kernel(f, m)
    def _nsub(self, n, dt, bg, row, nsub, tgt, non, cap):
        return self.lib.ref_nsub(n, dt, bg, row, nsub, tgt, non, cap)
    def _buckets(self, *a): return self.lib.ref_buckets(*a)

    def _dsa(self, prm, sh, n, mass, dunit, dt, mode, reacc, crp, cre, qpi, qepri, dis, nin):
        return self.lib.ref_dsa_inject(prm, sh, n, mass, dunit, dt, mode, reacc, crp, cre, qpi, qepri,
                                       dis, nin)

    def ic_emission(self, cre, nbins, z, nu_min, nu_max):
        """(fic [nbins][nb], eps [ncell][nbins]) from the reference's
        prepare_ic_kernel_flat and prepare_ic_emission_batch."""
        cre = np.ascontiguousarray(cre, dtype=np.float64)
        fic = np.empty((nbins, self.nb)); eps = np.empty((cre.shape[0], nbins))
        if self.lib.ref_ic_emission(cre.shape[0], nbins, z, nu_min, nu_max, cre, fic, eps) != 0:
            raise RuntimeError("ref_ic_emission failed")
        return fic, eps

    def synch_pitch_table(self, logy, w, logb_min, inv_dlogb, nlogb, xmin, logx_tab, logfx_tab, fx_tab):
        """The reference's prepare_synch_pitch_kernel_table on these arrays."""
        logy = np.ascontiguousarray(logy, np.float64)
        nfreq, _, nth = logy.shape
        out = np.empty((nlogb, nfreq, self.nb))
        if self.lib.ref_synch_pitch_table(nfreq, len(logx_tab), nth, nlogb, xmin, logb_min, inv_dlogb,
                                          _as_d(fx_tab), _as_d(logfx_tab), _as_d(logx_tab), logy,
                                          _as_d(w), out) != 0:
            raise RuntimeError("ref_synch_pitch_table failed")
        return out

    def synch_emission(self, cre, b_dyn, logb, logy, w, xmin, logx_tab, logfx_tab, fx_tab, table=None,
                       logb_min=0.0, inv_dlogb=0.0):
        """The reference's prepare_synch_emission_cell_major, with the pitch
        table when given, else through SYN_emissivity_from_arrays."""
        cre = np.ascontiguousarray(cre, np.float64)
        logy = np.ascontiguousarray(logy, np.float64)
        nfreq, _, nth = logy.shape
        nlogb = 0 if table is None else table.shape[0]
        tab = None if table is None else np.ascontiguousarray(table, np.float64)
        out = np.empty((cre.shape[0], nfreq))
        if self.lib.ref_synch_emission(cre.shape[0], nfreq, len(logx_tab), nth, nlogb, xmin, logb_min,
                                       inv_dlogb, _as_d(fx_tab), _as_d(logfx_tab), _as_d(logx_tab), logy,
                                       _as_d(w), _ptr(tab), _as_d(b_dyn), _as_d(logb), cre, out) != 0:
            raise RuntimeError("ref_synch_emission failed")
        return out

    def kernel_table(self, kind: str, nbins: int, lo: float, hi: float, z: float = 0.0):
        """prepare_{gamma,neutrino,ic}_kernel_flat: [nbins][nb]."""
        out = np.empty((nbins, self.nb))
        if kind == "gamma":
            rc = self.lib.ref_gamma_kernel_table(nbins, lo, hi, out)
        elif kind == "nu":
            rc = self.lib.ref_nu_kernel_table(nbins, lo, hi, out)
        else:
            rc = self.lib.ref_ic_kernel_table(nbins, lo, hi, z, out)
        if rc != 0:
            raise RuntimeError(f"ref kernel table {kind} failed")
        return out

    def hadronic_emission(self, kind: str, crp, n_gas, kern, lo: float, hi: float):
        """prepare_{gamma,neutrino}_emission_cell_major: [ncell][nbins]."""
        crp = np.ascontiguousarray(crp, np.float64)
        kern = np.ascontiguousarray(kern, np.float64)
        out = np.empty((crp.shape[0], kern.shape[0]))
        if self.lib.ref_hadronic_emission(0 if kind == "gamma" else 1, crp.shape[0], kern.shape[0], lo, hi,
                                          _as_d(n_gas), crp, kern, out) != 0:
            raise RuntimeError("ref hadronic emission failed")
        return out

    def synch_run(self, nfreq, nu_min, nu_max, ntheta, nlogb=512, logb_min=-6.0, logb_max=2.0,
                  b_field=None, cre=None, tables=True):
        """The reference's synchrotron tables (tracer_fp_synch_data_init_tables,
        tracer_fp_refresh_synch_kernel_table) and, given b_field and cre,
        prepare_synch_emission_cell_major.  Returns a dict of arrays."""
        nx = 2750
        r = {k: np.empty(nx) for k in ("logx", "logfx", "fx")}
        r["theta"], r["w"], r["nus"] = np.empty(ntheta), np.empty(ntheta), np.empty(nfreq)
        r["logy"] = np.empty((nfreq, self.nb, ntheta)) if tables else None
        r["table"] = np.empty((nlogb, nfreq, self.nb)) if tables else None
        ncell = 0 if cre is None else cre.shape[0]
        r["eps"] = np.empty((ncell, nfreq)) if ncell else None
        cre_c = None if cre is None else np.ascontiguousarray(cre, np.float64)
        b_c = None if b_field is None else np.ascontiguousarray(b_field, np.float64)
        outs = [r[k] for k in ("logx", "logfx", "fx", "theta", "w", "nus", "logy", "table", "eps")]
        rc = self.lib.ref_synch_run(nfreq, nu_min, nu_max, ntheta, nlogb, logb_min, logb_max, ncell,
                                    _ptr(b_c), _ptr(cre_c), *[_ptr(o) for o in outs])
        if rc != 0:
            raise RuntimeError(f"ref_synch_run failed: {rc}")
        return r

    def threads(self) -> int:
        return self.lib.ref_threads()

    def coeff_segments(self, nsub: int, allow_interp: bool) -> int:
        return self.lib.ref_coeff_segments(int(nsub), int(allow_interp))

    def cc_coeffs(self, dt, bg, rad_ic, rad_ic_m1, rad_ic_p1, mass=None, dis=None, crp=None, cre=None):
        n = bg.shape[1]; nb = self.nb
        outs = [np.empty(3 * n * nb) for _ in range(4)]
        err = self.lib.ref_cc_coeffs(n, dt, _as_d(bg), _as_d(rad_ic), _as_d(rad_ic_m1),
                                     _as_d(rad_ic_p1), _ptr(_as_d(mass)),
                                     _ptr(None if dis is None else np.ascontiguousarray(dis, np.uint8)),
                                     _ptr(_as_d(crp)), _ptr(_as_d(cre)), *outs)
        if err != 0:
            raise RuntimeError("ref cc_coeffs failed")
        return [o.reshape(3, n, nb) for o in outs]

    def evolve_segment(self, nstep, dt, windowed, on_start, on_end, bg, rad_ic, rad_ic_m1,
                       rad_ic_p1, qpi, qepri, crp, cre, mass=None, dis=None):
        n = bg.shape[1]
        err = self.lib.ref_evolve_segment(n, nstep, dt, int(windowed), on_start, on_end, _as_d(bg),
                                          _as_d(rad_ic), _as_d(rad_ic_m1), _as_d(rad_ic_p1),
                                          _as_d(qpi), _as_d(qepri), _ptr(_as_d(mass)),
                                          _ptr(None if dis is None else np.ascontiguousarray(dis, np.uint8)),
                                          crp, cre)
        if err != 0:
            raise RuntimeError("ref evolve_segment failed")

    def snapshot(self, bg_curr, bg_next, z_curr, z_next, allow, dt, elapsed, qpi, qepri, crp, cre,
                 mass=None, dis=None, ic=None):
        if ic is not None:
            raise ValueError("the reference computes its own IC rows")
        n = bg_curr.shape[1]
        nsub = np.empty(n, np.int32); non = np.empty(n, np.int32); bid = np.empty(n, np.int32)
        nbk = _i()
        m = _as_d(mass) if mass is not None else np.full(n, 1.0e7)
        err = self.lib.ref_snapshot(n, _as_d(bg_curr), _as_d(bg_next), z_curr, z_next, int(allow), dt,
                                    elapsed, _as_d(qpi), _as_d(qepri), _ptr(m),
                                    _ptr(None if dis is None else np.ascontiguousarray(dis, np.uint8)),
                                    crp, cre, nsub, non, bid, C.byref(nbk))
        if err != 0:
            raise RuntimeError(f"reference snapshot failed: {err}")
        return nsub, non, bid, nbk.value
