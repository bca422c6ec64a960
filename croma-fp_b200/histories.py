"""Tracer histories from the HDF5 snapshot series CROMA takes as input.

The reference reads a directory of snapshot files
``<tracer_file_dir>/<tracer_filename_base1>NNNN<tracer_file_extension>``
(params_tracer_10k.txt: ``tracer_10k/subset__tracer_z_dumpNNNN.h5``,
snapshots nsnp_i .. nsnp_f - 1) with libhdf5.  Here the files are read by
the library's own HDF5 reader (croma_b200_h5_*), and each snapshot's
background block is derived on the device (croma_b200_background_prepare):

* the timeline (read_redshift_hdf5, src/tracer_fp_background.c:70-146):
  z of every file's ``Redshift``; the next redshift of a snapshot is the
  following file's, the last one's is z - 0.01; the snapshot step is
  dz_to_dt(z - z_next, z) (src/COSFUNC.c:64-67) in the flat cosmology of
  src/COSFUNC.c:28-31 (H0 = 67.36, Omega_b + Omega_c of include/COSFUNC.h);
* the unit factors (tracer_init_hdf5_meta, :955-957): c_dens = dUnit,
  c_mag = sqrt(4 pi dUnit) vUnit;
* the raw fields (tracer_load_hdf5_raw_snapshot_slice, :1003-1204):
  temperature, density, B_x/y/z, div_v, curl_v, dx_phys;
* the background of snapshot i (the run loop, src/tracer_fp.c:917-1015):
  for i = 0 the raw fields of snapshot 0 as previous and current, no
  temperature floor and no curl interpolation; for i >= 1 snapshots i-1, i
  and i+1 (i again at the end), the temperature floor on, curl
  interpolation where a next snapshot exists;
* tracer masses: ``M_tracer`` of the first snapshot (variable_tracer_mass);
* the snapshot loop (include/tracer_fp_solve.inc): SnapshotSeries.evolve.
"""
from __future__ import annotations

import glob
import math
import os
import re

import numpy as np

from . import native

RAW_FIELDS = ("temperature", "density", "B_x", "B_y", "B_z", "div_v", "curl_v", "dx_phys")

# src/COSFUNC.c:24-31 with include/COSFUNC.h's defaults; src/CONSTANTS.c
H0 = 67.36
OM_B = 0.049301692328524445
OM_C = 0.26447041034523616
GYR = 3.1536e16
MPC = 3.0857e24


def hubble(z: float) -> float:
    """Hubble(z) in km/s/Mpc (src/COSFUNC.c:28-31)."""
    return H0 * math.sqrt((OM_C + OM_B) * math.pow(1.0 + z, 3.0) + (1.0 - (OM_C + OM_B)))


def dz_to_dt(dz: float, z: float) -> float:
    """Cosmic time in Gyr across a redshift step dz at z (src/COSFUNC.c:64-67)."""
    return dz / hubble(z) / (1.0 + z) / GYR * MPC * 1.0e-5


# the run parameters the background reads (src/params.c defaults; the
# tracer_10k run sets bfield_mode = max, eta_B = 0.05, mach_limit = 0.5)
DEFAULT_BACKGROUND = dict(bfield_mode=0, mu_mol=0.59, eta_B=0.05, mach_limit=0.5, l_turb_target_kpc=150.0)


def run_loop_raw(i: int, nsnap: int, raw_of, z, c_dens, c_mag) -> dict:
    """The CromaB200RawSnapshot fields of snapshot i of an nsnap-snapshot
    series as the run loop forms them (src/tracer_fp.c:917-1015): raw_of(k)
    gives snapshot k's raw fields (RAW_FIELDS), z / c_dens / c_mag its
    redshift and unit factors."""
    if i == 0:
        ip, ic, inx = 0, 0, (1 if nsnap > 1 else 0)
        floor, interp = 0, 0
    else:
        ip, ic, inx = i - 1, i, (i + 1 if i + 1 < nsnap else i)
        floor, interp = 1, int(i + 1 < nsnap)
    cur, prev, nxt = raw_of(ic), raw_of(ip), raw_of(inx)
    return dict(temp_K=cur["temperature"], density=cur["density"], bx=cur["B_x"], by=cur["B_y"], bz=cur["B_z"],
                div_v=cur["div_v"], curl_v_prev=prev["curl_v"], curl_v=cur["curl_v"], curl_v_next=nxt["curl_v"],
                l_turb_cm=cur["dx_phys"], c_dens=float(c_dens[ic]), c_mag=float(c_mag[ic]), z_prev=float(z[ip]),
                z_curr=float(z[ic]), z_next=float(z[inx]), apply_temp_floor=floor, allow_curl_interp=interp)


class SnapshotSeries:
    """The snapshot files base + NNNN + ext under directory, indices
    [first, last) (all present ones when not given), tracers
    [tracer_start, tracer_start + ntracer) of each."""

    def __init__(self, directory: str, base: str = "subset__tracer_z_dump", ext: str = ".h5",
                 first: int | None = None, last: int | None = None, tracer_start: int = 0,
                 ntracer: int | None = None, nb: int = 256):
        pat = re.compile(re.escape(base) + r"(\d+)" + re.escape(ext) + "$")
        found = {}
        for p in glob.glob(os.path.join(directory, base + "*" + ext)):
            m = pat.search(os.path.basename(p))
            if m:
                found[int(m.group(1))] = p
        if not found:
            raise FileNotFoundError(f"no snapshot files {base}NNNN{ext} under {directory}")
        lo = min(found) if first is None else first
        hi = max(found) + 1 if last is None else last
        missing = [k for k in range(lo, hi) if k not in found]
        if missing:
            raise FileNotFoundError(f"snapshot files missing for indices {missing[:5]}")
        self.index = list(range(lo, hi))
        self.files = [found[k] for k in self.index]
        self.nb = nb
        dims, _, _ = native.h5_shape(self.files[0], "density", nb)
        total = int(dims[0])
        self.tracer_start = tracer_start
        self.ntracer = (total - tracer_start) if ntracer is None else ntracer
        if tracer_start < 0 or self.ntracer <= 0 or tracer_start + self.ntracer > total:
            raise ValueError(f"tracers [{tracer_start}, {tracer_start + self.ntracer}) outside the {total} in the files")
        self.z = np.array([native.h5_read(f, "Redshift", nb=nb)[0] for f in self.files])
        self.c_dens = np.array([native.h5_read(f, "dUnit", nb=nb)[0] for f in self.files])
        self.c_velo = np.array([native.h5_read(f, "vUnit", nb=nb)[0] for f in self.files])
        self.c_mag = np.array([math.sqrt(4.0 * math.pi * cd) * cv for cd, cv in zip(self.c_dens, self.c_velo)])
        self.z_next = np.array([self.z[i + 1] if i + 1 < len(self.z) else self.z[i] - 0.01
                                for i in range(len(self.z))])
        self.dt = np.array([dz_to_dt(z - zn, z) for z, zn in zip(self.z, self.z_next)])
        self._raw: dict = {}

    def __len__(self):
        return len(self.files)

    def raw(self, i: int) -> dict:
        """The raw fields of snapshot i (cached)."""
        if i not in self._raw:
            self._raw[i] = {k: native.h5_read(self.files[i], k, self.tracer_start, self.ntracer, nb=self.nb)
                            for k in RAW_FIELDS}
        return self._raw[i]

    def mass(self) -> np.ndarray:
        """Tracer masses in M_sun (M_tracer of the first snapshot)."""
        return native.h5_read(self.files[0], "M_tracer", self.tracer_start, self.ntracer, nb=self.nb)

    def particle_ids(self, i: int = 0) -> np.ndarray:
        return native.h5_read(self.files[i], "particle_ID", self.tracer_start, self.ntracer, integer=True,
                              nb=self.nb)

    def raw_snapshot(self, i: int) -> dict:
        """The CromaB200RawSnapshot fields of snapshot i as the run loop forms them."""
        return run_loop_raw(i, len(self.files), self.raw, self.z, self.c_dens, self.c_mag)

    def background(self, i: int, params: dict | None = None, ctx=None) -> np.ndarray:
        """The [8][ntracer] background of snapshot i, derived on the device."""
        return native.background_prepare(self.raw_snapshot(i), params or DEFAULT_BACKGROUND, ctx=ctx, nb=self.nb)

    def evolve(self, fp, start: int = 0, stop: int | None = None, params: dict | None = None,
               elapsed: float = 0.0, background=None, before=None, after=None) -> float:
        """Advance the tracers fp holds (a native.TracerFP over this series'
        tracers, or anything with its snapshot method) through snapshots
        [start, stop) as the reference's snapshot loop does
        (include/tracer_fp_solve.inc:1-20, :1676-1779): snapshot i goes from
        background i to background i + 1 over dt[i], interpolating between
        them; the series' last snapshot has no next one and runs on its own
        background with z_next = z and no interpolation; elapsed (Gyr)
        accumulates dt.  background(i) gives snapshot i's [8][ntracer] block
        (default: derived on the device with params); before(i, bg) runs
        before snapshot i with its background, on the spectra the snapshot
        starts from (where the reference computes the emission,
        include/tracer_fp_solve.inc:117-426); after(i, elapsed) runs after
        snapshot i.  Returns the elapsed time.  Shock fields are not
        read: the tracer_10k run has DSA off (params_tracer_10k.txt:70-72)."""
        n = len(self)
        stop = n if stop is None else stop
        if not 0 <= start <= stop <= n:
            raise ValueError(f"snapshots [{start}, {stop}) outside the series' {n}")
        if start == stop:
            return elapsed
        bg_of = background if background is not None else (lambda i: self.background(i, params))
        curr = bg_of(start)
        for i in range(start, stop):
            has_next = i + 1 < n
            nxt = bg_of(i + 1) if has_next else curr
            z_next = float(self.z[i + 1]) if has_next else float(self.z[i])
            if before is not None:
                before(i, curr)
            fp.snapshot(curr, nxt, float(self.z[i]), z_next, has_next, float(self.dt[i]), elapsed)
            elapsed += float(self.dt[i])
            if after is not None:
                after(i, elapsed)
            curr = nxt
        return elapsed
