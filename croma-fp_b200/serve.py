"""ctypes front-end of the request server (include/croma_b200_serve.h).

    srv = Server(cfg, hbm_budget_gb=120, max_concurrent=4)
    rid = srv.submit(bg, z, dt, crp_in, cre_in, species_mask=3)
    srv.wait(rid); crp, cre = srv.output(rid)

Host arrays handed to submit are kept alive here until the request is
collected with output() / forget().
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native

_d, _i, _vp, _ll = C.c_double, C.c_int, C.c_void_p, C.c_longlong
QUEUED, RUNNING, DONE, FAILED, CANCELLED = range(5)
STATES = ("queued", "running", "done", "failed", "cancelled")


class ServeConfig(C.Structure):
    _fields_ = [("base", native.CromaB200Config), ("device", _i), ("hbm_budget_bytes", _d),
                ("max_concurrent", _i), ("workspace_bytes_per_request", _d)]


class Request(C.Structure):
    _fields_ = [("ntracer", _i), ("species_mask", _i), ("nsnap", _i), ("bg", _vp),
                ("bg_field_stride", _ll), ("bg_snap_stride", _ll), ("z", _vp), ("dt_snap", _vp),
                ("elapsed0_gyr", _d), ("crp_in", _vp), ("cre_in", _vp), ("mass_msun", _vp),
                ("crp_out", _vp), ("cre_out", _vp)]


def _lib(nb):
    L = native.load_library(nb)
    if not getattr(L, "_serve_bound", False):
        P = C.POINTER
        L.croma_b200_serve_create.argtypes = [P(ServeConfig), P(_vp)]
        L.croma_b200_serve_destroy.argtypes = [_vp]
        L.croma_b200_serve_request_bytes.argtypes = [_vp, _i]
        L.croma_b200_serve_request_bytes.restype = _d
        L.croma_b200_serve_submit.argtypes = [_vp, P(Request)]
        L.croma_b200_serve_submit.restype = _ll
        L.croma_b200_serve_poll.argtypes = [_vp, _ll]
        L.croma_b200_serve_wait.argtypes = [_vp, _ll, _d]
        L.croma_b200_serve_cancel.argtypes = [_vp, _ll]
        L.croma_b200_serve_result.argtypes = [_vp, _ll, P(_i), P(_d), P(_d), C.c_char_p, _i]
        L.croma_b200_serve_stats.argtypes = [_vp, P(_i), P(_i), P(_d), P(_i), P(_d), P(_d)]
        L._serve_bound = True
    return L


class ServeError(RuntimeError):
    pass


class Server:
    def __init__(self, cfg, hbm_budget_gb: float = 120.0, max_concurrent: int = 4,
                 workspace_gb_per_request: float = 4.0, path: str = "fused", device: int = 0):
        self.nb = cfg.nb
        self.lib = _lib(cfg.nb)
        sc = ServeConfig()
        sc.base = native.make_config(cfg, path)
        sc.device = device
        sc.hbm_budget_bytes = hbm_budget_gb * 1e9
        sc.max_concurrent = max_concurrent
        sc.workspace_bytes_per_request = workspace_gb_per_request * 1e9
        h = _vp()
        if self.lib.croma_b200_serve_create(C.byref(sc), C.byref(h)) != 0:
            raise ServeError(self.lib.croma_b200_last_error().decode())
        self.h = h
        self._keep = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.croma_b200_serve_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def request_bytes(self, ntracer: int) -> float:
        return self.lib.croma_b200_serve_request_bytes(self.h, int(ntracer))

    def submit(self, bg, z, dt, crp_in=None, cre_in=None, mass=None, species_mask=3,
               elapsed0=0.0, field_stride=0, snap_stride=0, ntracer=None) -> int:
        """bg: [nsnap+1][8][ntracer] (or a strided view base with the strides
        given in doubles); returns the request id."""
        bg = np.asarray(bg)
        z = np.ascontiguousarray(z, dtype=np.float64)
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        n = int(ntracer if ntracer is not None else bg.shape[-1])
        nsnap = dt.size
        out_p = np.empty((n, self.nb)); out_e = np.empty((n, self.nb))
        keep = [bg, z, dt, out_p, out_e]
        r = Request()
        r.ntracer, r.species_mask, r.nsnap = n, int(species_mask), nsnap
        r.bg = bg.ctypes.data
        r.bg_field_stride, r.bg_snap_stride = int(field_stride), int(snap_stride)
        r.z, r.dt_snap, r.elapsed0_gyr = z.ctypes.data, dt.ctypes.data, float(elapsed0)
        for name, a in (("crp_in", crp_in), ("cre_in", cre_in), ("mass_msun", mass)):
            if a is not None:
                a = np.ascontiguousarray(a, dtype=np.float64)
                keep.append(a)
                setattr(r, name, a.ctypes.data)
        r.crp_out, r.cre_out = out_p.ctypes.data, out_e.ctypes.data
        rid = self.lib.croma_b200_serve_submit(self.h, C.byref(r))
        if rid < 0:
            raise ServeError(f"{rid}: {self.lib.croma_b200_last_error().decode()}")
        self._keep[rid] = keep
        return rid

    def poll(self, rid: int) -> int:
        return self.lib.croma_b200_serve_poll(self.h, rid)

    def wait(self, rid: int, timeout_s: float = -1.0) -> int:
        return self.lib.croma_b200_serve_wait(self.h, rid, float(timeout_s))

    def cancel(self, rid: int) -> int:
        return self.lib.croma_b200_serve_cancel(self.h, rid)

    def result(self, rid: int):
        """(rc, latency_s, run_s, message) of a finished request."""
        rc, lat, run = _i(), _d(), _d()
        msg = C.create_string_buffer(512)
        if self.lib.croma_b200_serve_result(self.h, rid, C.byref(rc), C.byref(lat), C.byref(run), msg, 512):
            raise ServeError(self.lib.croma_b200_last_error().decode())
        return rc.value, lat.value, run.value, msg.value.decode()

    def output(self, rid: int):
        """Final (crp, cre) of a finished request; releases its buffers."""
        keep = self._keep.pop(rid)
        return keep[3], keep[4]

    def forget(self, rid: int):
        self._keep.pop(rid, None)

    def stats(self):
        q, r, c = _i(), _i(), _i()
        b, p50, p99 = _d(), _d(), _d()
        self.lib.croma_b200_serve_stats(self.h, C.byref(q), C.byref(r), C.byref(b), C.byref(c),
                                        C.byref(p50), C.byref(p99))
        return dict(queued=q.value, running=r.value, bytes_in_use=b.value, completed=c.value,
                    p50_s=p50.value, p99_s=p99.value)
