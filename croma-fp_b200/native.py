"""ctypes binding of the native C ABI (include/croma_b200.h) and a small
Python front end, ``TracerFP``, that runs snapshots through it.

The library must be built first (``python croma-fp_b200/build.py`` or
``__graft_entry__.build()``); loading fails loudly when it is missing or
when no CUDA device is present -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .config import RunConfig

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

PATHS = {"plain": 0, "fused": 1, "fp32r": 2}

_d, _i, _vp = C.c_double, C.c_int, C.c_void_p


class CromaB200Config(C.Structure):
    _fields_ = [("nb", _i), ("species_mask", _i), ("pmin", _d), ("pmax", _d), ("pemin", _d),
                ("pemax", _d), ("dpp_model", _i), ("ttd_tacc_model", _i), ("t_acc_direct_gyr", _d),
                ("mach_limit", _d), ("psi", _d), ("eta_dpp_cap", _d), ("nsub_safety", _d),
                ("nsub_max", _i), ("coeff_interp_min_steps", _i), ("coeff_interp_max_segments", _i),
                ("reacc_window_mode", _i), ("f_eddy", _d), ("t_off_gyr", _d), ("t_acc_off_gyr", _d),
                ("path", _i)]


class CromaB200Snapshot(C.Structure):
    _fields_ = [("bg_curr", _vp), ("bg_next", _vp), ("bg_on_device", _i), ("z_curr", _d),
                ("z_next", _d), ("allow_interp", _i), ("dt_snap", _d), ("elapsed_gyr", _d)]


class CromaB200RawSnapshot(C.Structure):
    _fields_ = [("temp_K", _vp), ("density", _vp), ("bx", _vp), ("by", _vp), ("bz", _vp), ("div_v", _vp),
                ("curl_v_prev", _vp), ("curl_v", _vp), ("curl_v_next", _vp), ("l_turb_cm", _vp),
                ("c_dens", _d), ("c_mag", _d), ("z_prev", _d), ("z_curr", _d), ("z_next", _d),
                ("apply_temp_floor", _i), ("allow_curl_interp", _i)]


class CromaB200BackgroundParams(C.Structure):
    _fields_ = [("bfield_mode", _i), ("mu_mol", _d), ("eta_B", _d), ("mach_limit", _d),
                ("l_turb_target_kpc", _d)]


_LIBS: dict = {}


def library_path(nb: int) -> str:
    return os.path.join(LIBDIR, f"libcroma_b200_np{nb}.so")


def load_library(nb: int) -> C.CDLL:
    if nb in _LIBS:
        return _LIBS[nb]
    path = library_path(nb)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python croma-fp_b200/build.py {nb}`")
    L = C.CDLL(path)
    P = C.POINTER
    L.croma_b200_last_error.restype = C.c_char_p
    L.croma_b200_create.argtypes = [P(CromaB200Config), _i, P(_vp)]
    L.croma_b200_destroy.argtypes = [_vp]
    L.croma_b200_reserve.argtypes = [_vp, _i]
    L.croma_b200_set_state.argtypes = [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp]
    L.croma_b200_get_state.argtypes = [_vp, _vp, _vp]
    L.croma_b200_snapshot.argtypes = [_vp, P(CromaB200Snapshot), _i]
    L.croma_b200_snapshot_host.argtypes = [_vp, P(CromaB200Snapshot), _i, _vp, _vp, _vp, _i]
    L.croma_b200_set_workspace_limit.argtypes = [_vp, _d]
    L.croma_b200_set_priority.argtypes = [_vp, _i]
    L.croma_b200_get_schedule.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp, _vp]
    L.croma_b200_ic_row.argtypes = [_vp, _d, _vp]
    L.croma_b200_get_grid.argtypes = [_vp, _i, _vp]
    L.croma_b200_get_secondary_kernel.argtypes = [_vp, _vp, _vp]
    L.croma_b200_stream.argtypes = [_vp]
    L.croma_b200_stream.restype = _vp
    L.croma_b200_sync.argtypes = [_vp]
    L.croma_b200_state_device.argtypes = [_vp, P(_vp), P(_vp)]
    L.croma_b200_last_launch_count.argtypes = [_vp]
    L.croma_b200_set_kernel_timing.argtypes = [_vp, _i]
    L.croma_b200_kernel_stats.argtypes = [_vp, _i, P(_d), P(C.c_longlong)]
    L.croma_b200_reset_kernel_stats.argtypes = [_vp]
    L.croma_b200_fp64_peak.argtypes = [P(_d)]
    L.croma_b200_rcp_check.argtypes = [C.c_longlong, _vp, _vp]
    L.croma_b200_exp_check.argtypes = [C.c_longlong, _vp, _vp]
    L.croma_b200_h5_shape.argtypes = [C.c_char_p, C.c_char_p, P(_i), P(C.c_longlong), _i, P(_i), P(_i)]
    L.croma_b200_h5_read_f64.argtypes = [C.c_char_p, C.c_char_p, C.c_longlong, C.c_longlong, _vp]
    L.croma_b200_h5_read_i64.argtypes = [C.c_char_p, C.c_char_p, C.c_longlong, C.c_longlong, _vp]
    L.croma_b200_background_prepare.argtypes = [_vp, _i, P(CromaB200RawSnapshot), P(CromaB200BackgroundParams),
                                                _i, _vp]
    L.croma_b200_get_sources.argtypes = [_vp, _vp, _vp, _vp]
    L.croma_b200_set_state_broadcast.argtypes = [_vp, _i, _vp, _vp, _d]
    L.croma_b200_set_dsa.argtypes = [_vp, P(CromaB200DsaParams)]
    L.croma_b200_dsa_inject.argtypes = [_vp, P(CromaB200Shocks), _d, _d, _i, _i, P(_i)]
    L.croma_b200_emission_ic.argtypes = [_vp, _i, _vp, _vp, P(_d)]
    L.croma_b200_emission_hadronic.argtypes = [_vp, _i, _d, _d, _vp, _vp, _vp, _vp, P(_d)]
    L.croma_b200_emission_synch.argtypes = [_vp, _i, _i, _d, _d, _vp, _vp, _vp, _vp, P(_d)]
    L.croma_b200_emission_setup.argtypes = [_vp, P(CromaB200EmissionSetup)]
    L.croma_b200_emission_run.argtypes = [_vp, _vp, _d, _vp, _vp, _vp, _vp, _i]
    L.croma_b200_emission_table.argtypes = [_vp, _i, _vp]
    L.croma_b200_step_host.argtypes = [_vp, P(CromaB200Snapshot), P(CromaB200StepHost)]
    L.croma_b200_host_alloc.argtypes = [C.c_size_t, P(_vp)]
    L.croma_b200_get_tuning.argtypes = [_vp, _i, P(_i), P(_i), P(_i), P(_d)]
    L.croma_b200_host_free.argtypes = [_vp]
    _LIBS[nb] = L
    return L


class CromaB200EmissionSetup(C.Structure):
    _fields_ = [("nfreq", _i), ("nu_min_s", _d), ("nu_max_s", _d), ("ntheta_pitch", _i), ("nlogb", _i),
                ("logb_min", _d), ("logb_max", _d), ("nbins_ic", _i), ("nu_min_ic", _d), ("nu_max_ic", _d),
                ("nbins_gamma", _i), ("egamma_min", _d), ("egamma_max", _d), ("nbins_nu", _i),
                ("enu_min", _d), ("enu_max", _d)]


# The emission bands of the full-pipeline workload: synchrotron at 64
# frequencies over 10 MHz .. 10 GHz; IC, gamma and neutrinos at 64 energies
# over 1 keV .. 1 PeV (IC in log10 Hz: E / h); the reference's default pitch
# angles (512) and log-B table (512 planes over [-6, 2]).
EMISSION_CONFIG4 = dict(nfreq=64, nu_min_s=7.0, nu_max_s=10.0, ntheta_pitch=512, nlogb=512, logb_min=-6.0,
                        logb_max=2.0, nbins_ic=64, nu_min_ic=17.383, nu_max_ic=29.383, nbins_gamma=64,
                        egamma_min=-6.0, egamma_max=6.0, nbins_nu=64, enu_min=-6.0, enu_max=6.0)


class CromaB200DsaParams(C.Structure):
    _fields_ = [("eta_model_initial", _i), ("eta_model_reacc", _i), ("chi_p", _d), ("chi_e", _d),
                ("k_ep", _d), ("pmax_p_mc", _d), ("pmax_e_mc", _d), ("min_mach", _d),
                ("gamma_gas", _d), ("xcr_pmin_pmc", _d), ("reacc_eta_cap", _d), ("mu_mol", _d),
                ("pmin_dsa_p_log10", _d), ("pmin_dsa_e_log10", _d), ("inject_species", _i)]


SHOCK_FIELDS = ("mach", "prestemp", "presden", "pre_density_cgs", "upstream_speed_cgs",
                "shock_side_code", "dsa_trigger", "dsa_mach", "dsa_pre_density", "dsa_flux_cgs")


class CromaB200Shocks(C.Structure):
    _fields_ = [(n, _vp) for n in SHOCK_FIELDS] + [("has_dsa", _i), ("on_device", _i)]


class CromaB200StepHost(C.Structure):
    _fields_ = [("shocks", C.POINTER(CromaB200Shocks)), ("dsa_mode", _i), ("dsa_reacc", _i),
                ("density_unit", _d), ("eps_syn", _vp), ("eps_ic", _vp), ("eps_gamma", _vp), ("eps_nu", _vp),
                ("crp_out", _vp), ("cre_out", _vp)]


class CromaError(RuntimeError):
    pass


def make_config(cfg: RunConfig, path: str = "plain") -> CromaB200Config:
    """CromaB200Config from a RunConfig."""
    c = CromaB200Config()
    for name, _ in CromaB200Config._fields_:
        if name == "dpp_model":
            c.dpp_model = cfg.dpp_model_id()
        elif name == "species_mask":
            c.species_mask = cfg.species_mask()
        elif name == "path":
            c.path = PATHS[path]
        else:
            setattr(c, name, getattr(cfg, name))
    return c


def fp64_peak(nb: int = 256) -> float:
    """FP64 FMA throughput of the current device in TFLOP/s (measured live)."""
    L = load_library(nb)
    t = _d()
    if L.croma_b200_fp64_peak(C.byref(t)) != 0:
        raise CromaError(L.croma_b200_last_error().decode())
    return t.value


def h5_shape(path: str, dataset: str, nb: int = 256):
    """(dims tuple, 'float' | 'int', element bytes) of an HDF5 dataset."""
    L = load_library(nb)
    rank, cls, size = _i(), _i(), _i()
    dims = (C.c_longlong * 32)()
    if L.croma_b200_h5_shape(path.encode(), dataset.encode(), C.byref(rank), dims, 32, C.byref(cls),
                             C.byref(size)) != 0:
        raise CromaError(L.croma_b200_last_error().decode())
    return tuple(dims[i] for i in range(rank.value)), ("float" if cls.value == 1 else "int"), size.value


def h5_read(path: str, dataset: str, offset: int = 0, count=None, integer: bool = False, nb: int = 256):
    """Elements [offset, offset + count) of an HDF5 dataset as float64 (or
    int64 for integer=True); count None reads to the end."""
    L = load_library(nb)
    dims, _, _ = h5_shape(path, dataset, nb)
    n = int(np.prod(dims)) if dims else 1
    if count is None:
        count = n - offset
    out = np.empty(count, np.int64 if integer else np.float64)
    fn = L.croma_b200_h5_read_i64 if integer else L.croma_b200_h5_read_f64
    if fn(path.encode(), dataset.encode(), int(offset), int(count), _p(out)) != 0:
        raise CromaError(L.croma_b200_last_error().decode())
    return out


def background_prepare(raw: dict, params: dict, ctx=None, nb: int = 256, on_device: bool = False, out=None):
    """croma_b200_background_prepare: the [8][ntracer] background block from
    one snapshot's raw fields.  raw maps the CromaB200RawSnapshot fields to
    arrays (host, or device addresses with on_device) and scalars; params the
    CromaB200BackgroundParams fields.  Returns the host block (or None when
    out is a device address)."""
    L = load_library(nb)
    r = CromaB200RawSnapshot()
    keep = []
    n = None
    for name, typ in CromaB200RawSnapshot._fields_:
        v = raw.get(name)
        if typ is _vp:
            if v is None:
                setattr(r, name, None)
            elif on_device:
                setattr(r, name, int(v))
            else:
                a = _c(v)
                keep.append(a)
                n = a.shape[0] if n is None else n
                if a.shape != (n,):
                    raise ValueError(f"raw field {name} must be [ntracer]")
                setattr(r, name, a.ctypes.data)
        else:
            setattr(r, name, v if v is not None else 0)
    if on_device:
        n = int(raw["ntracer"])
    prm = CromaB200BackgroundParams(**params)
    if n is None:
        raise ValueError("raw has no per-tracer field")
    if out is None:
        if on_device:
            raise ValueError("on_device needs an output address")
        out = np.empty((8, n))
    elif not on_device and (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (8, n)
                            or not out.flags.c_contiguous or not out.flags.writeable):
        raise ValueError(f"out must be a writeable C-contiguous float64 array of shape (8, {n})")
    dst = out if on_device else out.ctypes.data
    h = ctx.h if ctx is not None else None
    rc = L.croma_b200_background_prepare(h, n, C.byref(r), C.byref(prm), int(bool(on_device)), dst)
    if rc != 0:
        raise CromaError(L.croma_b200_last_error().decode())
    return None if on_device else out


def _math_check(fn: str, x, nb: int):
    L = load_library(nb)
    xa = _c(x)
    out = np.empty_like(xa)
    if getattr(L, fn)(xa.size, _p(xa), _p(out)) != 0:
        raise CromaError(L.croma_b200_last_error().decode())
    return out


def rcp_check(x, nb: int = 256):
    """The device reciprocal of the factor and per-step kernels applied to
    the float64 array x (croma_b200_rcp_check)."""
    return _math_check("croma_b200_rcp_check", x, nb)


def exp_check(x, nb: int = 256):
    """The factor kernels' table-driven exponential applied to the float64
    array x (croma_b200_exp_check)."""
    return _math_check("croma_b200_exp_check", x, nb)


def _shocks_struct(shocks: dict):
    """CromaB200Shocks from a dict of SHOCK_FIELDS arrays (or device
    addresses with shocks['on_device']); returns (struct, arrays to keep)."""
    sh = CromaB200Shocks()
    keep = []
    on_dev = int(shocks.get("on_device", 0))
    for n in SHOCK_FIELDS:
        a = shocks.get(n)
        if a is None:
            continue
        if on_dev:
            setattr(sh, n, int(a))
        else:
            arr = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(arr)
            setattr(sh, n, arr.ctypes.data)
    sh.has_dsa = int(shocks.get("has_dsa", 0))
    sh.on_device = on_dev
    return sh, keep


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def _c(a, dtype=np.float64):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


class PinnedArray:
    """A float64 numpy array in page-locked host memory of exactly its size
    (croma_b200_host_alloc); .a is the array, .free() releases it."""

    def __init__(self, shape, nb: int = 512):
        self.lib = load_library(nb)
        n = int(np.prod(shape))
        ptr = _vp()
        if self.lib.croma_b200_host_alloc(C.c_size_t(n * 8), C.byref(ptr)) != 0:
            raise CromaError(self.lib.croma_b200_last_error().decode())
        self.ptr = ptr.value
        buf = (C.c_double * n).from_address(self.ptr)
        self.a = np.frombuffer(buf, dtype=np.float64).reshape(shape)

    def free(self):
        if self.ptr:
            self.a = None
            self.lib.croma_b200_host_free(self.ptr)
            self.ptr = None


class TracerFP:
    """One device-resident batch of tracers advanced snapshot by snapshot."""

    def __init__(self, cfg: RunConfig, path: str = "plain", device: int = 0):
        self.cfg = cfg
        self.nb = cfg.nb
        self.lib = load_library(cfg.nb)
        c = make_config(cfg, path)
        h = _vp()
        self._check(self.lib.croma_b200_create(C.byref(c), device, C.byref(h)))
        self.h = h
        self.ntracer = 0

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.croma_b200_last_error().decode()
            raise CromaError(f"croma_b200 call failed ({rc}): {msg}")

    def set_workspace_limit(self, nbytes: float):
        """Cap on the evolve workspace (takes effect at the next reserve /
        set_state with a new tracer count); tracers beyond it run in chunks."""
        self._check(self.lib.croma_b200_set_workspace_limit(self.h, float(nbytes)))

    def set_priority(self, priority: int):
        """CUDA stream priority of the context's stream (lower runs first)."""
        self._check(self.lib.croma_b200_set_priority(self.h, int(priority)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.croma_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ----------------------------------------------------------
    def set_state(self, crp, cre, qpi=None, qepri=None, mass=None, dis=None):
        crp, cre = _c(crp), _c(cre)
        n = crp.shape[0]
        qpi, qepri, mass = _c(qpi), _c(qepri), _c(mass)
        dis = _c(dis, np.uint8)
        self._check(self.lib.croma_b200_set_state(self.h, n, _p(crp), _p(cre), _p(qpi), _p(qepri),
                                                  _p(mass), _p(dis)))
        self.ntracer = n

    def set_state_broadcast(self, ntracer: int, crp_row, cre_row, mass: float = 1.0e7):
        """Every tracer from the same seed rows [nb]."""
        a, b = _c(crp_row), _c(cre_row)
        self._check(self.lib.croma_b200_set_state_broadcast(self.h, int(ntracer), _p(a), _p(b), float(mass)))
        self.ntracer = int(ntracer)

    def get_state(self, crp=None, cre=None):
        """Spectra as cell-major host arrays; crp / cre may be given (e.g.
        page-locked buffers) to be filled in place."""
        if crp is None:
            crp = np.empty((self.ntracer, self.nb))
        if cre is None:
            cre = np.empty((self.ntracer, self.nb))
        for a in (crp, cre):
            if a.shape != (self.ntracer, self.nb) or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("state buffers must be C-contiguous float64 [ntracer][nb]")
        self._check(self.lib.croma_b200_get_state(self.h, _p(crp), _p(cre)))
        return crp, cre

    def state_device(self):
        a, b = _vp(), _vp()
        self._check(self.lib.croma_b200_state_device(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # -- snapshots ------------------------------------------------------
    def snapshot(self, bg_curr, bg_next, z_curr, z_next, allow, dt, elapsed, sync=True):
        """Advance one snapshot.  bg_* are host arrays [8][ntracer] or device
        addresses (ints)."""
        s = CromaB200Snapshot()
        if isinstance(bg_curr, int):
            s.bg_curr, s.bg_next, s.bg_on_device = bg_curr, bg_next, 1
            keep = None
        else:
            bc = _c(bg_curr)
            bn = _c(bg_next) if bg_next is not None else bc
            keep = (bc, bn)
            s.bg_curr, s.bg_next, s.bg_on_device = bc.ctypes.data, bn.ctypes.data, 0
        s.z_curr, s.z_next, s.allow_interp = z_curr, z_next, int(bool(allow))
        s.dt_snap, s.elapsed_gyr = dt, elapsed
        self._check(self.lib.croma_b200_snapshot(self.h, C.byref(s), int(bool(sync))))
        del keep

    def snapshot_host(self, crp, cre, bg_curr, bg_next, z_curr, z_next, allow, dt, elapsed, mass=None,
                      chunks=0):
        """One snapshot from host spectra to host spectra with the copies
        overlapped with the evolve (croma_b200_snapshot_host).  crp / cre are
        C-contiguous float64 [ntracer][nb] host arrays, overwritten in place
        with the evolved spectra (page-locked ones let the copies overlap);
        bg_* are host arrays [8][ntracer]."""
        for a in (crp, cre):
            if a.ndim != 2 or a.shape[1] != self.nb or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("state buffers must be C-contiguous float64 [ntracer][nb]")
        if crp.shape != cre.shape:
            raise ValueError("crp and cre must have the same shape")
        n = crp.shape[0]
        m = _c(mass)
        if m is not None and m.shape != (n,):
            raise ValueError("mass must have one value per tracer")
        bc = _c(bg_curr)
        bn = _c(bg_next) if bg_next is not None else bc
        if bc.size != 8 * n or bn.size != 8 * n:
            raise ValueError("backgrounds must be [8][ntracer]")
        s = CromaB200Snapshot()
        s.bg_curr, s.bg_next, s.bg_on_device = bc.ctypes.data, bn.ctypes.data, 0
        s.z_curr, s.z_next, s.allow_interp = z_curr, z_next, int(bool(allow))
        s.dt_snap, s.elapsed_gyr = dt, elapsed
        self._check(self.lib.croma_b200_snapshot_host(self.h, C.byref(s), n, _p(crp), _p(cre), _p(m),
                                                      int(chunks)))
        self.ntracer = n

    def step_host(self, bg_curr, bg_next, z_curr, z_next, allow, dt, elapsed, shocks=None, dsa_mode="off",
                  dsa_reacc="off", density_unit=1.0, outputs=None):
        """One snapshot step through host memory (croma_b200_step_host): DSA
        from host shock fields, emission and evolve; outputs maps 'syn', 'ic',
        'gamma', 'nu', 'crp', 'cre' to host arrays filled in place (page-locked
        ones let the copies overlap)."""
        outputs = outputs or {}
        bc = _c(bg_curr)
        bn = _c(bg_next) if bg_next is not None else bc
        snap = CromaB200Snapshot()
        snap.bg_curr, snap.bg_next, snap.bg_on_device = bc.ctypes.data, bn.ctypes.data, 0
        snap.z_curr, snap.z_next, snap.allow_interp = z_curr, z_next, int(bool(allow))
        snap.dt_snap, snap.elapsed_gyr = dt, elapsed
        io = CromaB200StepHost()
        keep = None
        if shocks is not None:
            sh, keep = _shocks_struct(shocks)
            io.shocks = C.pointer(sh)
        io.dsa_mode = self.DSA_MODES[dsa_mode] if isinstance(dsa_mode, str) else int(dsa_mode)
        io.dsa_reacc = self.DSA_REACC[dsa_reacc] if isinstance(dsa_reacc, str) else int(dsa_reacc)
        io.density_unit = float(density_unit)
        for k, f in (("syn", "eps_syn"), ("ic", "eps_ic"), ("gamma", "eps_gamma"), ("nu", "eps_nu"),
                     ("crp", "crp_out"), ("cre", "cre_out")):
            a = outputs.get(k)
            if a is not None:
                if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape[0] != self.ntracer:
                    raise ValueError(f"output {k} must be C-contiguous float64 with one row per tracer")
                setattr(io, f, a.ctypes.data)
        self._check(self.lib.croma_b200_step_host(self.h, C.byref(snap), C.byref(io)))
        del keep

    SOLVERS = {0: "thomas-scan", 1: "thomas-scan-fp32-refined", 2: "pcr", 3: "thomas-scan-smem",
               4: "thomas-scan-rhs-smem", 5: "thomas-scan4"}
    VARIANTS = ("scan x1", "scan x2", "smem scan x1", "smem scan x2", "pcr x1", "rhs scan x1", "rhs scan x2",
                "scan4 x1", "scan4 x2")

    def tuning(self, species: int):
        """The steps-kernel autotuner's record for species 0 (protons) or 1
        (electrons): dict(tuned, solver, warps_per_block, variant_ms)."""
        t, so, w = _i(), _i(), _i()
        ms = (_d * len(self.VARIANTS))()
        self._check(self.lib.croma_b200_get_tuning(self.h, species, C.byref(t), C.byref(so), C.byref(w), ms))
        return {"tuned": t.value, "solver": self.SOLVERS.get(so.value, so.value), "warps_per_block": w.value,
                "variant_ms": {n: (m if m >= 0 else None) for n, m in zip(self.VARIANTS, list(ms))}}

    def sync(self):
        self._check(self.lib.croma_b200_sync(self.h))

    def schedule(self):
        n = self.ntracer
        out = {k: np.empty(n, np.int32) for k in ("nsub", "non", "target", "bucket_ids", "bucket_indices")}
        nb = np.zeros(1, np.int32)
        self._check(self.lib.croma_b200_get_schedule(self.h, _p(out["nsub"]), _p(out["non"]),
                                                     _p(out["target"]), _p(out["bucket_ids"]),
                                                     _p(out["bucket_indices"]), _p(nb)))
        out["nbuckets"] = int(nb[0])
        return out

    # -- tables ---------------------------------------------------------
    def ic_row(self, z):
        out = np.empty(self.nb + 2)
        self._check(self.lib.croma_b200_ic_row(self.h, z, _p(out)))
        return out[:self.nb], out[self.nb], out[self.nb + 1]

    def grid(self, species):
        out = np.empty(3 * self.nb + 2)
        self._check(self.lib.croma_b200_get_grid(self.h, species, _p(out)))
        n = self.nb
        return out[:n], out[n:2 * n], out[2 * n:3 * n], out[3 * n], out[3 * n + 1]

    def secondary_kernel(self):
        f = np.empty((self.nb, self.nb))
        m = np.empty(self.nb, np.int32)
        self._check(self.lib.croma_b200_get_secondary_kernel(self.h, _p(f), _p(m)))
        return f, m

    def stream(self) -> int:
        return self.lib.croma_b200_stream(self.h) or 0

    def last_launch_count(self) -> int:
        return self.lib.croma_b200_last_launch_count(self.h)

    # -- emissivities of the resident spectra ---------------------------
    def emission_ic(self, fic):
        """IC emissivity [ntracer][nbands] of the resident electron spectra;
        fic [nbands][nb].  Returns (eps, device ms)."""
        f = _c(fic)
        if f.ndim != 2 or f.shape[1] != self.nb:
            raise ValueError("fic must be [nbands][nb]")
        eps, ms = np.empty((self.ntracer, f.shape[0])), _d()
        self._check(self.lib.croma_b200_emission_ic(self.h, f.shape[0], _p(f), _p(eps), C.byref(ms)))
        return eps, ms.value

    def emission_hadronic(self, kernel, n_gas, beta_p, e_min, e_max):
        """Gamma or neutrino emissivity [ntracer][nbins] of the resident
        proton spectra (kernel [nbins][nb] chooses which).  Returns (eps, ms)."""
        k, n, b = _c(kernel), _c(n_gas), _c(beta_p)
        if k.ndim != 2 or k.shape[1] != self.nb:
            raise ValueError("kernel must be [nbins][nb]")
        if n.shape != (self.ntracer,) or b.shape != (self.nb,):
            raise ValueError("n_gas must be [ntracer] and beta_p [nb]")
        eps, ms = np.empty((self.ntracer, k.shape[0])), _d()
        self._check(self.lib.croma_b200_emission_hadronic(self.h, k.shape[0], e_min, e_max, _p(n), _p(b), _p(k),
                                                          _p(eps), C.byref(ms)))
        return eps, ms.value

    def emission_synch(self, table, b_dyn, logb, logb_min, inv_dlogb):
        """Synchrotron emissivity [ntracer][nfreq] of the resident electron
        spectra through the pitch-kernel table [nlogb][nfreq][nb]."""
        t, bd, lb = _c(table), _c(b_dyn), _c(logb)
        if t.ndim != 3 or t.shape[2] != self.nb:
            raise ValueError("table must be [nlogb][nfreq][nb]")
        if bd.shape != (self.ntracer,) or lb.shape != (self.ntracer,):
            raise ValueError("b_dyn and logb must be [ntracer]")
        eps, ms = np.empty((self.ntracer, t.shape[1])), _d()
        self._check(self.lib.croma_b200_emission_synch(self.h, t.shape[1], t.shape[0], logb_min, inv_dlogb, _p(t),
                                                       _p(bd), _p(lb), _p(eps), C.byref(ms)))
        return eps, ms.value

    # -- emission into device or host memory ---------------------------
    def emission_setup(self, **kw):
        """Builds the emission tables on the device (croma_b200_emission_setup);
        keywords are the CromaB200EmissionSetup fields, missing ones 0."""
        st = CromaB200EmissionSetup()
        for name, _ in CromaB200EmissionSetup._fields_:
            setattr(st, name, kw.get(name, 0))
        self._check(self.lib.croma_b200_emission_setup(self.h, C.byref(st)))
        self._emis = {n: kw.get(n, 0) for n in ("nfreq", "nbins_ic", "nbins_gamma", "nbins_nu")}

    def emission_run(self, bg, z, kinds=("syn", "ic", "gamma", "nu")):
        """Emissivities of the resident spectra from a host background
        [8][ntracer]: dict kind -> [ntracer][bins]."""
        b = _c(bg)
        if b.shape != (8, self.ntracer):
            raise ValueError("bg must be [8][ntracer]")
        cols = dict(syn=self._emis["nfreq"], ic=self._emis["nbins_ic"], gamma=self._emis["nbins_gamma"],
                    nu=self._emis["nbins_nu"])
        out = {k: np.empty((self.ntracer, cols[k])) for k in kinds if cols[k] > 0}
        self._check(self.lib.croma_b200_emission_run(self.h, _p(b), float(z), _p(out.get("syn")), _p(out.get("ic")),
                                                     _p(out.get("gamma")), _p(out.get("nu")), 0))
        return out

    def emission_run_device(self, bg_ptr: int, z, syn=0, ic=0, gamma=0, nu=0):
        """Asynchronous emission on device pointers (ints, 0 skips a kind)."""
        self._check(self.lib.croma_b200_emission_run(self.h, bg_ptr, float(z), syn or None, ic or None,
                                                     gamma or None, nu or None, 1))

    def emission_table(self, which: str, shape):
        out = np.empty(shape)
        self._check(self.lib.croma_b200_emission_table(self.h, {"synch": 0, "ic": 1}[which], _p(out)))
        return out

    KERNEL_KINDS = {"evolve": 0, "coeff": 1, "secondary": 2}

    def set_kernel_timing(self, enable: bool):
        self._check(self.lib.croma_b200_set_kernel_timing(self.h, int(bool(enable))))

    def kernel_stats(self, kind: str):
        ms, n = _d(), C.c_longlong()
        self._check(self.lib.croma_b200_kernel_stats(self.h, self.KERNEL_KINDS[kind], C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def get_sources(self):
        """(qpi, qepri, disable_adiabatic) as cell-major host arrays."""
        qpi = np.empty((self.ntracer, self.nb)); qe = np.empty((self.ntracer, self.nb))
        dis = np.empty(self.ntracer, np.uint8)
        self._check(self.lib.croma_b200_get_sources(self.h, _p(qpi), _p(qe), _p(dis)))
        return qpi, qe, dis

    def set_dsa(self, params):
        """params: an object with the CromaB200DsaParams field names
        (config.DsaParams)."""
        p = CromaB200DsaParams()
        for name, _ in CromaB200DsaParams._fields_:
            setattr(p, name, getattr(params, name))
        self._check(self.lib.croma_b200_set_dsa(self.h, C.byref(p)))

    DSA_MODES = {"off": 0, "tracer_state": 1, "tracer_source": 2}
    DSA_REACC = {"off": 0, "positive_delta": 1, "drury83": 2}

    def dsa_inject(self, shocks: dict, density_unit: float, dt_gyr: float, mode, reacc="off") -> int:
        """One snapshot's shock injection; shocks maps SHOCK_FIELDS names to
        host arrays [ntracer] (or device addresses with shocks['on_device'])
        plus 'has_dsa'.  Returns the number of tracers injected."""
        sh, keep = _shocks_struct(shocks)
        m = self.DSA_MODES[mode] if isinstance(mode, str) else int(mode)
        r = self.DSA_REACC[reacc] if isinstance(reacc, str) else int(reacc)
        nin = _i()
        self._check(self.lib.croma_b200_dsa_inject(self.h, C.byref(sh), float(density_unit), float(dt_gyr),
                                                   m, r, C.byref(nin)))
        return nin.value

    def reset_kernel_stats(self):
        self._check(self.lib.croma_b200_reset_kernel_stats(self.h))
