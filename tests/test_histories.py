"""Real tracer histories (HDF5 tracer input), on the CPU.

* The library's HDF5 reader (croma_b200_h5_*) on the reference's own
  tracer_10k snapshot series, where the reference tree is present
  (CROMA_REFERENCE_ROOT): every file opens, every field the background reads
  has one element per tracer, the tracer ids agree across the series, the
  redshifts fall by 0.01 per file from 1, the fields are finite and the
  positive ones positive, a scalar reads as one element, and damaged or
  foreign files are refused with an error instead of a crash.
* The background restatement (oracle/croma_oracle_background.c) is pinned
  bit for bit to the reference's own prepare_background_cell (oracle/_ref)
  on those files, and to the committed fixture golden_histories.npz
  (tests/golden/make_golden.py) everywhere.
"""
import json
import os
import shutil

import numpy as np
import pytest

from conftest import ROOT, load_package
from golden_io import GOLDEN_DIR

load_package()
from croma_fp_b200 import config, histories, native  # noqa: E402

import sys  # noqa: E402
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle  # noqa: E402

REF = os.environ.get("CROMA_REFERENCE_ROOT", "/root/reference")
SERIES = os.path.join(REF, "tracer_10k")
FIX = np.load(os.path.join(GOLDEN_DIR, "golden_histories.npz"))
PRM = json.loads(str(FIX["params"]))
have_series = pytest.mark.skipif(not os.path.isdir(SERIES), reason="reference tracer series not present")


def fixture_raw(i):
    keys = ("temp_K", "density", "bx", "by", "bz", "div_v", "curl_v_prev", "curl_v", "curl_v_next", "l_turb_cm",
            "c_dens", "c_mag", "z_prev", "z_curr", "z_next", "apply_temp_floor", "allow_curl_interp")
    raw = {k: FIX[f"s{i}_{k}"] for k in keys}
    for k in ("c_dens", "c_mag", "z_prev", "z_curr", "z_next"):
        raw[k] = float(raw[k])
    for k in ("apply_temp_floor", "allow_curl_interp"):
        raw[k] = int(raw[k])
    return raw


@have_series
def test_reader_on_the_reference_snapshot_series():
    S = histories.SnapshotSeries(SERIES)
    assert len(S) == 100 and S.index[0] == 25 and S.ntracer == 10000
    assert np.allclose(S.z, 1.0 - 0.01 * np.arange(100), atol=2e-5)
    assert np.all(np.diff(S.z) < 0) and np.all(S.dt > 0) and np.all(S.c_dens > 0) and np.all(S.c_mag > 0)
    ids0 = S.particle_ids(0)
    assert len(np.unique(ids0)) == S.ntracer
    for i in (0, 1, 50, 99):
        assert np.array_equal(S.particle_ids(i), ids0)
        raw = S.raw(i)
        for k, v in raw.items():
            assert v.shape == (S.ntracer,) and np.all(np.isfinite(v)), k
        for k in ("temperature", "density", "dx_phys"):
            assert np.all(raw[k] > 0), k
    f = S.files[0]
    assert native.h5_shape(f, "Redshift") == ((), "float", 8)
    assert native.h5_shape(f, "particle_ID") == ((10000,), "int", 8)
    # a slice equals the same elements of the whole dataset
    whole = native.h5_read(f, "density")
    assert np.array_equal(native.h5_read(f, "density", 1234, 777), whole[1234:1234 + 777])
    m = S.mass()
    assert np.all((m >= 1e7) & (m <= 1e9))


@have_series
def test_reader_refuses_damaged_and_foreign_files(tmp_path):
    src = histories.SnapshotSeries(SERIES, first=25, last=26).files[0]
    with pytest.raises(native.CromaError, match="no dataset or group"):
        native.h5_read(src, "no_such_field")
    with pytest.raises(native.CromaError):
        native.h5_read(src, "density", 9990, 20)   # past the end
    with pytest.raises(native.CromaError, match="not an integer dataset"):
        native.h5_read(src, "density", integer=True)
    data = open(src, "rb").read()
    for cut in (16, 700, 6000, len(data) // 2):   # truncated copies: headers or data cut off
        p = tmp_path / f"cut{cut}.h5"
        p.write_bytes(data[:cut])
        with pytest.raises(native.CromaError):
            native.h5_read(str(p), "z_coordinate")
    p = tmp_path / "foreign.h5"
    p.write_bytes(b"not an HDF5 file" * 100)
    with pytest.raises(native.CromaError, match="not an HDF5 file"):
        native.h5_shape(str(p), "density")
    # a corrupted B-tree signature
    bad = bytearray(data)
    pos = bad.find(b"TREE")
    bad[pos:pos + 4] = b"XXXX"
    p = tmp_path / "badtree.h5"
    p.write_bytes(bytes(bad))
    with pytest.raises(native.CromaError, match="B-tree"):
        native.h5_read(str(p), "density")
    shutil.rmtree(tmp_path, ignore_errors=True)


@have_series
@pytest.mark.skipif(not pyoracle.reference_available(128), reason="oracle/_ref not built")
def test_background_restatement_matches_reference_on_the_series():
    S = histories.SnapshotSeries(SERIES, first=25, last=125, ntracer=3000)
    for i in (0, 1, 57, 99):   # first snapshot (no floor, no interpolation), middle, last (no next)
        raw = S.raw_snapshot(i)
        for prm in (PRM, dict(PRM, bfield_mode=1), dict(PRM, bfield_mode=2, mach_limit=0.0)):
            assert np.array_equal(pyoracle.background(raw, prm), pyoracle.reference_background(raw, prm)), (i, prm)


def test_background_restatement_matches_fixture():
    for i in FIX["snaps"]:
        assert np.array_equal(pyoracle.background(fixture_raw(int(i)), PRM), FIX[f"s{int(i)}_bg_ref"]), i


def test_background_curl_interpolation_and_floor():
    """A zero curl_v is interpolated in z between the neighbours when allowed,
    and the temperature floor lifts T below 1e4 K (prepare_background_cell,
    src/fp_shared_core.c:883-892)."""
    raw = fixture_raw(1)
    raw = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in raw.items()}
    raw["curl_v"][:8] = 0.0
    raw["temp_K"][8:16] = 5.0e3
    bg = pyoracle.background(raw, PRM)
    off = pyoracle.background(dict(raw, allow_curl_interp=0, apply_temp_floor=0), PRM)
    assert np.all(bg[5, :8] != off[5, :8])                       # dv from the interpolated curl
    assert np.allclose(bg[1, 8:16], 8.62e-5 * 1.0e4 * 1.0e-9, rtol=1e-15)
    assert np.allclose(off[1, 8:16], 8.62e-5 * 5.0e3 * 1.0e-9, rtol=1e-15)


def test_timeline_restates_the_reference_cosmology():
    """dt of a snapshot = dz / H(z) / (1 + z) in Gyr (src/COSFUNC.c:64-67):
    the step between z = 1 and 0.99 is about 41 Myr and within 1 % of the
    exact cosmic-time integral over the step."""
    z0, z1 = 1.0, 0.99
    dt = histories.dz_to_dt(z0 - z1, z0)
    zs = np.linspace(z1, z0, 20001)
    f = 1.0 / ((1.0 + zs) * np.array([histories.hubble(z) for z in zs]))
    exact = np.trapezoid(f, zs) / histories.GYR * histories.MPC * 1.0e-5
    assert 0.035 < dt < 0.045 and abs(dt / exact - 1.0) < 0.01
    cfg = config.tracer_10k()
    assert cfg.species == "electron_only" and cfg.reacc_window_mode == 1 and cfg.eta_dpp_cap == 0.1


@have_series
@pytest.mark.skipif(not pyoracle.reference_available(128), reason="oracle/_ref not built")
def test_oracle_evolves_real_histories_like_the_reference():
    """Ten consecutive snapshots of 24 real tracers (every 400th of the
    series) with the reference's tracer_10k settings: the oracle on its own
    backgrounds and the reference's compiled code on the reference's
    backgrounds agree bit for bit, nsub included."""
    from croma_fp_b200 import synth
    cfg = config.tracer_10k(nb=128)
    S = histories.SnapshotSeries(SERIES, first=40, last=51)
    idx = np.arange(0, S.ntracer, 400)
    o, ref = pyoracle.Oracle(cfg), pyoracle.ReferenceCPU(cfg)
    gp, ge = o.grid(0), o.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), len(idx), cfg.species)
    mass = np.ascontiguousarray(S.mass()[idx])
    q = np.zeros_like(crp)
    a = [crp.copy(), cre.copy()]
    b = [crp.copy(), cre.copy()]
    elapsed = 0.0

    def bg(i, fn):
        raw = S.raw_snapshot(i)
        sel = {k: (np.ascontiguousarray(v[idx]) if isinstance(v, np.ndarray) else v) for k, v in raw.items()}
        return fn(sel, PRM)

    for i in range(1, 10):
        args_o = (bg(i, pyoracle.background), bg(i + 1, pyoracle.background))
        args_r = (bg(i, pyoracle.reference_background), bg(i + 1, pyoracle.reference_background))
        common = (float(S.z[i]), float(S.z[i + 1]), True, float(S.dt[i]), elapsed)
        n_o = o.snapshot(*args_o, *common, q, q, a[0], a[1], mass=mass)[0]
        n_r = ref.snapshot(*args_r, *common, q, q, b[0], b[1], mass=mass)[0]
        elapsed += float(S.dt[i])
        assert np.array_equal(n_o, n_r) and np.array_equal(a[1], b[1]), i
    assert np.any(a[1] != cre)


def test_series_loader_and_snapshot_loop_on_a_written_series(tmp_path):
    """The fixture's 20 snapshots written as a snapshot series (series_io),
    read back through SnapshotSeries: redshifts, snapshot steps, unit
    factors, raw fields and masses are the fixture's.  evolve() runs the
    reference's snapshot loop: its calls (backgrounds, z_next, interpolation
    flag, dt, elapsed) over the series' end, and on the oracle over five
    snapshots the same spectra, bit for bit, as the loop written out by hand
    (the real-history GPU tests' form)."""
    import series_io
    series_io.write_series(str(tmp_path))
    n = series_io.NLONG
    S = histories.SnapshotSeries(str(tmp_path), nb=128)
    assert len(S) == n and S.ntracer == 64 and S.index[0] == series_io.FIRST
    assert np.array_equal(S.z, FIX["z"][:n])
    assert np.array_equal(S.dt[:n - 1], FIX["dt"][:n - 1])   # the last step differs: the series ends there
    assert np.array_equal(S.c_dens, FIX["c_dens"][:n])
    assert np.allclose(S.c_mag, FIX["c_mag"][:n], rtol=1e-15, atol=0.0)
    for k in (0, 7, n - 1):
        raw = S.raw(k)
        for f in histories.RAW_FIELDS:
            assert np.array_equal(raw[f], FIX[f"long{k}_{f}"]), (k, f)
    assert np.array_equal(S.mass(), FIX["long_mass"])
    assert np.array_equal(S.particle_ids(3), np.arange(100, 164))

    calls = []

    class Recorder:
        def snapshot(self, bc, bn, z, zn, allow, dt, elapsed):
            calls.append((bc, bn, z, zn, allow, dt, elapsed))

    blocks = {i: np.full((8, 64), float(i)) for i in range(n)}
    seen = []
    end = S.evolve(Recorder(), start=n - 3, background=blocks.__getitem__, elapsed=1.0,
                   before=lambda i, bg: seen.append((i, bg, len(calls))))
    assert [(i, bg is blocks[i], k) for i, bg, k in seen] == [(n - 3, True, 0), (n - 2, True, 1), (n - 1, True, 2)]
    assert [c[0] is blocks[i] for c, i in zip(calls, range(n - 3, n))] == [True] * 3
    assert calls[0][1] is blocks[n - 2] and calls[0][3] == S.z[n - 2] and calls[0][4] is True
    assert calls[-1][1] is blocks[n - 1] and calls[-1][3] == calls[-1][2] == S.z[n - 1] and calls[-1][4] is False
    assert [c[5] for c in calls] == [float(S.dt[i]) for i in range(n - 3, n)]
    assert calls[1][6] == 1.0 + float(S.dt[n - 3])
    assert end == (1.0 + float(S.dt[n - 3])) + float(S.dt[n - 2]) + float(S.dt[n - 1])
    with pytest.raises(ValueError):
        S.evolve(Recorder(), start=3, stop=2)

    from croma_fp_b200 import synth
    cfg = config.tracer_10k(nb=128)
    S16 = histories.SnapshotSeries(str(tmp_path), nb=128, ntracer=16)
    mass = S16.mass()
    o = pyoracle.Oracle(cfg)
    gp, ge = o.grid(0), o.grid(1)
    crp0, cre0 = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 16, cfg.species)
    q = np.zeros_like(crp0)

    class OracleFP:
        def __init__(self):
            self.crp, self.cre = crp0.copy(), cre0.copy()

        def snapshot(self, bc, bn, z, zn, allow, dt, elapsed):
            o.snapshot(bc, bn, z, zn, allow, dt, elapsed, q, q, self.crp, self.cre, mass=mass)

    bg = [pyoracle.background(S16.raw_snapshot(i), PRM) for i in range(6)]
    a = OracleFP()
    S16.evolve(a, stop=5, background=bg.__getitem__)
    b = OracleFP()
    elapsed = 0.0
    for k in range(5):
        b.snapshot(bg[k], bg[k + 1], float(S16.z[k]), float(S16.z[k + 1]), True, float(S16.dt[k]), elapsed)
        elapsed += float(S16.dt[k])
    assert np.array_equal(a.cre, b.cre) and np.any(a.cre != cre0)


def test_series_refuses_gaps_and_tracer_ranges_outside_the_files(tmp_path):
    """A missing snapshot file inside the requested range, a directory without
    snapshot files, and a tracer range past the files' tracers are refused
    before anything is read past them."""
    import os as _os
    import series_io
    paths = series_io.write_series(str(tmp_path), nsnap=4)
    S = histories.SnapshotSeries(str(tmp_path), first=26, last=28, nb=128)
    assert S.index == [26, 27] and len(S) == 2 and S.ntracer == 64
    with pytest.raises(ValueError, match="outside"):
        histories.SnapshotSeries(str(tmp_path), tracer_start=60, ntracer=8, nb=128)
    _os.remove(paths[2])
    with pytest.raises(FileNotFoundError, match="missing"):
        histories.SnapshotSeries(str(tmp_path), nb=128)
    assert len(histories.SnapshotSeries(str(tmp_path), last=27, nb=128)) == 2
    empty = tmp_path / "empty"
    empty.mkdir()
    with pytest.raises(FileNotFoundError, match="no snapshot files"):
        histories.SnapshotSeries(str(empty), nb=128)


@pytest.mark.skipif(not pyoracle.reference_available(128), reason="oracle/_ref not built")
def test_nonpositive_density_refused_like_the_reference():
    """A tracer with zero density: the reference's prepare_background_cell
    fails on it (src/fp_shared_core.c:866-932 returns -1), and the
    restatement refuses the block too (the device path reports -2 with the
    tracer's fields zeroed, tests/test_gpu_histories.py)."""
    raw = fixture_raw(1)
    raw = {k: (v[:8].copy() if isinstance(v, np.ndarray) else v) for k, v in raw.items()}
    raw["density"][2] = 0.0
    with pytest.raises(RuntimeError, match="tracer 2"):
        pyoracle.reference_background(raw, PRM)
    with pytest.raises(RuntimeError, match="-2"):
        pyoracle.background(raw, PRM)
