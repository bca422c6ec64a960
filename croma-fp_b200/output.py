"""Output files and checkpoints in the reference's formats
(include/croma_b200_output.h; src/tracer_fp_output.c and
src/tracer_fp_restart.c of the reference) through ctypes.

    out = OutputFile(nb, "/data/run", "CRE", rank=0, mode="tile", nslab=nsnap + 1, nrow=ntracer, ncol=nb)
    out.write(0, cre0)                          # host rows
    out.write_state(fp, slab=k + 1)             # straight from a TracerFP's resident spectra
    out.close()
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native

_i, _d, _vp, _sz, _l = C.c_int, C.c_double, C.c_void_p, C.c_size_t, C.c_long
MODES = {"tile": 0, "mapped": 1}


class Checkpoint(C.Structure):
    _fields_ = [("dir", C.c_char_p), ("mpi_rank", _i), ("world_size", _i), ("ntracer", _i),
                ("ntracer_global", _i), ("nsnap", _i), ("nfreq", _i), ("nsnp_i", _i), ("nsnp_f", _i),
                ("completed_snapshot", _i), ("tracer_start", _l), ("tracer_ids", _vp)]


def _lib(nb: int):
    L = native.load_library(nb)
    if not getattr(L, "_output_bound", False):
        L.croma_b200_output_open.argtypes = [C.c_char_p, C.c_char_p, _i, _i, _sz, _sz, _sz, _i, C.POINTER(_vp)]
        L.croma_b200_output_write.argtypes = [_vp, _sz, _vp, _vp, _vp, _i]
        L.croma_b200_output_write_state.argtypes = [_vp, _vp, _vp, _sz, _vp, _i]
        L.croma_b200_output_flush.argtypes = [_vp]
        L.croma_b200_output_close.argtypes = [_vp]
        P = C.POINTER(Checkpoint)
        L.croma_b200_checkpoint_write_host.argtypes = [P, _i, _i, _vp, _vp]
        L.croma_b200_checkpoint_read_host.argtypes = [P, _i, _i, _vp, _vp, C.POINTER(_i)]
        L.croma_b200_checkpoint_write.argtypes = [_vp, P]
        L.croma_b200_checkpoint_read.argtypes = [_vp, P, C.POINTER(_i)]
        L._output_bound = True
    return L


class OutputError(RuntimeError):
    pass


def _check(L, rc):
    if rc != 0:
        raise OutputError(f"{L.croma_b200_last_error().decode()} (code {rc})")


def _p(a):
    return None if a is None else a.ctypes.data


def _rows(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != shape:
        raise ValueError(f"expected an array of shape {shape}, got {a.shape}")
    return a


class OutputFile:
    """One output file of one rank (tile or mapped layout)."""

    def __init__(self, nb: int, directory: str, stem: str, rank: int, mode: str, nslab: int, nrow: int,
                 ncol: int, resume_existing: bool = False):
        self.L = _lib(nb)
        self.nrow, self.ncol = int(nrow), int(ncol)
        h = _vp()
        _check(self.L, self.L.croma_b200_output_open(directory.encode(), stem.encode(), int(rank), MODES[mode],
                                                     int(nslab), self.nrow, self.ncol, int(bool(resume_existing)),
                                                     C.byref(h)))
        self.h = h

    def write(self, slab: int, rows, rho=None, mass=None, per_cc: bool = False):
        rows = _rows(rows, (self.nrow, self.ncol))
        rho = None if rho is None else _rows(rho, (self.nrow,))
        mass = None if mass is None else _rows(mass, (self.nrow,))
        _check(self.L, self.L.croma_b200_output_write(self.h, int(slab), _p(rows), _p(rho), _p(mass),
                                                      int(bool(per_cc))))

    @staticmethod
    def write_state(fp: "native.TracerFP", cre_out: "OutputFile", crp_out: "OutputFile | None", slab: int,
                    rho=None, per_cc: bool = False):
        """Queue slab `slab` of fp's resident spectra (asynchronous)."""
        rho = None if rho is None else _rows(rho, (cre_out.nrow,))
        _check(cre_out.L, cre_out.L.croma_b200_output_write_state(fp.h, cre_out.h,
                                                                  None if crp_out is None else crp_out.h,
                                                                  int(slab), _p(rho), int(bool(per_cc))))

    def flush(self):
        _check(self.L, self.L.croma_b200_output_flush(self.h))

    def close(self):
        if self.h:
            h, self.h = self.h, None
            _check(self.L, self.L.croma_b200_output_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _ckpt(directory, rank, world, ntracer_global, nsnap, nfreq, nsnp_i, nsnp_f, tracer_start, ids,
          completed=0):
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    ck = Checkpoint(directory.encode(), int(rank), int(world), ids.size, int(ntracer_global), int(nsnap),
                    int(nfreq), int(nsnp_i), int(nsnp_f), int(completed), int(tracer_start), ids.ctypes.data)
    return ck, ids


def checkpoint_write_host(nb: int, directory: str, crp, cre, ids, *, rank=0, world=1, ntracer_global=None,
                          nsnap=1, nfreq=0, nsnp_i=0, nsnp_f=0, tracer_start=0, completed=0):
    L = _lib(nb)
    crp = np.ascontiguousarray(crp, dtype=np.float64)
    cre = np.ascontiguousarray(cre, dtype=np.float64)
    ck, keep = _ckpt(directory, rank, world, ntracer_global or len(ids), nsnap, nfreq, nsnp_i, nsnp_f,
                     tracer_start, ids, completed)
    _check(L, L.croma_b200_checkpoint_write_host(C.byref(ck), crp.shape[1], cre.shape[1], _p(crp), _p(cre)))


def checkpoint_read_host(nb: int, directory: str, ids, *, np_bins=None, npe_bins=None, rank=0, world=1,
                         ntracer_global=None, nsnap=1, nfreq=0, nsnp_i=0, nsnp_f=0, tracer_start=0):
    L = _lib(nb)
    np_bins = np_bins or nb
    npe_bins = npe_bins or nb
    ck, keep = _ckpt(directory, rank, world, ntracer_global or len(ids), nsnap, nfreq, nsnp_i, nsnp_f,
                     tracer_start, ids)
    crp = np.empty((len(ids), np_bins))
    cre = np.empty((len(ids), npe_bins))
    done = _i()
    _check(L, L.croma_b200_checkpoint_read_host(C.byref(ck), np_bins, npe_bins, _p(crp), _p(cre), C.byref(done)))
    return crp, cre, done.value


def checkpoint_write(fp: "native.TracerFP", directory: str, ids, **kw):
    L = _lib(fp.nb)
    ck, keep = _ckpt(directory, kw.get("rank", 0), kw.get("world", 1), kw.get("ntracer_global") or len(ids),
                     kw.get("nsnap", 1), kw.get("nfreq", 0), kw.get("nsnp_i", 0), kw.get("nsnp_f", 0),
                     kw.get("tracer_start", 0), ids, kw.get("completed", 0))
    _check(L, L.croma_b200_checkpoint_write(fp.h, C.byref(ck)))


def checkpoint_read(fp: "native.TracerFP", directory: str, ids, **kw) -> int:
    L = _lib(fp.nb)
    ck, keep = _ckpt(directory, kw.get("rank", 0), kw.get("world", 1), kw.get("ntracer_global") or len(ids),
                     kw.get("nsnap", 1), kw.get("nfreq", 0), kw.get("nsnp_i", 0), kw.get("nsnp_f", 0),
                     kw.get("tracer_start", 0), ids)
    done = _i()
    _check(L, L.croma_b200_checkpoint_read(fp.h, C.byref(ck), C.byref(done)))
    fp.ntracer = len(ids)
    return done.value
