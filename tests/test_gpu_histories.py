"""Real tracer histories on the GPU (HDF5 tracer input): the device background
(croma_b200_background_prepare) of the committed tracer_10k fixture
(tests/golden/golden_histories.npz: the reference's own
prepare_background_cell outputs), and those tracers evolved with it over
three snapshots (both paths) and over twenty (on-chip path), against the
oracle evolving the same tracers on the reference's (or its own)
backgrounds.

The device background repeats the reference's operations in its order
without contraction; only pow(L_target / L, 0.3333) comes from CUDA's libm,
so the fields that do not depend on it (n_gas, kT, div v, L_turb, c_s) are
bit-identical and the rest agree to a few ulp."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, load_package
from golden_io import GOLDEN_DIR, rel_err

load_package()
from croma_fp_b200 import config, native, synth  # noqa: E402

import sys  # noqa: E402
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle  # noqa: E402

pytestmark = pytest.mark.gpu

FIX = np.load(os.path.join(GOLDEN_DIR, "golden_histories.npz"))
PRM = json.loads(str(FIX["params"]))
KEYS = ("temp_K", "density", "bx", "by", "bz", "div_v", "curl_v_prev", "curl_v", "curl_v_next", "l_turb_cm",
        "c_dens", "c_mag", "z_prev", "z_curr", "z_next", "apply_temp_floor", "allow_curl_interp")


def raw(i, sel=slice(None)):
    r = {}
    for k in KEYS:
        v = FIX[f"s{i}_{k}"]
        if v.ndim:
            r[k] = np.ascontiguousarray(v[sel])
        else:
            r[k] = int(v) if k in ("apply_temp_floor", "allow_curl_interp") else float(v)
    return r


def test_device_background_matches_reference():
    for i in FIX["snaps"]:
        i = int(i)
        got = native.background_prepare(raw(i), PRM)
        ref = FIX[f"s{i}_bg_ref"]
        for f in (0, 1, 3, 4, 6):
            assert np.array_equal(got[f], ref[f]), (i, f)
        assert float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300))) <= 1e-14, i


@pytest.mark.parametrize("prm", [dict(bfield_mode=1), dict(bfield_mode=2, mach_limit=0.0),
                                 dict(bfield_mode=0, l_turb_target_kpc=40.0, mu_mol=0.6)])
def test_device_background_matches_restatement_in_every_field_mode(prm):
    """The B-field modes (simulation field, dynamo field, the larger of the
    two), no Mach limit and another turbulence scale and molecular weight:
    the device background against the oracle's restatement (itself bit-exact
    to the reference's prepare_background_cell) on the fixture's first and
    middle snapshots."""
    p = dict(PRM, **prm)
    for i in (0, 2):
        got = native.background_prepare(raw(i), p)
        ref = pyoracle.background(raw(i), p)
        for f in (0, 1, 3, 4, 6):
            assert np.array_equal(got[f], ref[f]), (i, f)
        assert float(np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300))) <= 1e-14, i


def test_device_pointers_equal_host_call():
    torch = pytest.importorskip("torch")
    r = raw(2)
    host = native.background_prepare(r, PRM)
    dev = {k: (torch.from_numpy(v).cuda() if isinstance(v, np.ndarray) else v) for k, v in r.items()}
    out = torch.empty((8, host.shape[1]), dtype=torch.float64, device="cuda")
    addr = {k: (v.data_ptr() if hasattr(v, "data_ptr") else v) for k, v in dev.items()}
    addr["ntracer"] = host.shape[1]
    native.background_prepare(addr, PRM, on_device=True, out=out.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), host)


def test_nonpositive_density_is_reported():
    r = raw(1, slice(0, 16))
    r["density"] = r["density"].copy()
    r["density"][3] = 0.0
    with pytest.raises(native.CromaError, match="density <= 0"):
        native.background_prepare(r, PRM)


@pytest.mark.parametrize("path", ["fused", "plain"])
def test_real_histories_evolve_like_the_oracle(path):
    """64 tracers of the real series, electron_only as the reference's
    tracer_10k run configures them (config.tracer_10k), three snapshots from
    the start of the series: the GPU on its own device backgrounds, the
    oracle on the reference's."""
    cfg = config.tracer_10k(nb=128)
    n = 64
    sel = slice(0, n)
    mass = np.ascontiguousarray(FIX["mass"][sel])
    fp = native.TracerFP(cfg, path=path)
    o = pyoracle.Oracle(cfg)
    try:
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        fp.set_state(crp, cre, mass=mass)
        o_crp, o_cre = crp.copy(), cre.copy()
        q = np.zeros_like(crp)
        dev_bg = [native.background_prepare(raw(k, sel), PRM) for k in range(4)]
        ref_bg = [np.ascontiguousarray(FIX[f"s{k}_bg_ref"][:, sel]) for k in range(4)]
        z, dt = FIX["z"], FIX["dt"]
        elapsed = 0.0
        for k in range(3):
            fp.snapshot(dev_bg[k], dev_bg[k + 1], float(z[k]), float(z[k + 1]), True, float(dt[k]), elapsed,
                        sync=True)
            o.snapshot(ref_bg[k], ref_bg[k + 1], float(z[k]), float(z[k + 1]), True, float(dt[k]), elapsed,
                       q, q, o_crp, o_cre, mass=mass)
            elapsed += float(dt[k])
            g_crp, g_cre = fp.get_state()
            assert rel_err(g_cre, o_cre) <= 1e-10, k
            assert np.any(g_cre != cre)
    finally:
        fp.close()


def test_real_histories_over_twenty_snapshots():
    """The fixture's first 64 tracers over the first 20 snapshots of the
    series (treated as a 20-snapshot run), on-chip FP64 path on the device
    backgrounds against the oracle on its own: within the FP64 bar after
    every snapshot, so no error builds up along real histories."""
    from croma_fp_b200 import histories
    cfg = config.tracer_10k(nb=128)
    nlong = 20
    raw_of = lambda k: {f: FIX[f"long{k}_{f}"] for f in histories.RAW_FIELDS}   # noqa: E731
    z, dt, c_dens, c_mag = FIX["z"], FIX["dt"], FIX["c_dens"], FIX["c_mag"]
    mass = np.ascontiguousarray(FIX["long_mass"])
    n = mass.shape[0]
    fp = native.TracerFP(cfg, path="fused")
    o = pyoracle.Oracle(cfg)
    try:
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        fp.set_state(crp, cre, mass=mass)
        o_crp, o_cre = crp.copy(), cre.copy()
        q = np.zeros_like(crp)
        raws = [histories.run_loop_raw(k, nlong, raw_of, z, c_dens, c_mag) for k in range(nlong)]
        dev_bg = [native.background_prepare(r, PRM) for r in raws]
        ora_bg = [pyoracle.background(r, PRM) for r in raws]
        elapsed = 0.0
        worst = 0.0
        for k in range(nlong - 1):
            fp.snapshot(dev_bg[k], dev_bg[k + 1], float(z[k]), float(z[k + 1]), True, float(dt[k]), elapsed,
                        sync=True)
            o.snapshot(ora_bg[k], ora_bg[k + 1], float(z[k]), float(z[k + 1]), True, float(dt[k]), elapsed,
                       q, q, o_crp, o_cre, mass=mass)
            elapsed += float(dt[k])
            g_crp, g_cre = fp.get_state()
            err = rel_err(g_cre, o_cre)
            worst = max(worst, err)
            assert err <= 1e-10, (k, err)
        print("worst over 19 snapshots", worst)
    finally:
        fp.close()


def test_snapshot_series_from_files(tmp_path):
    """End to end from files: the fixture's 20 snapshots written as a
    snapshot series (series_io), read by the library's HDF5 reader, each
    snapshot's background derived on the device, and the 64 tracers evolved
    on the GPU through all 20 snapshots by SnapshotSeries.evolve (the last
    one without a next snapshot), against the oracle running the same loop on
    its background restatement: within the FP64 bar after every snapshot."""
    import series_io
    from croma_fp_b200 import histories
    series_io.write_series(str(tmp_path))
    S = histories.SnapshotSeries(str(tmp_path), nb=128)
    cfg = config.tracer_10k(nb=128)
    n = S.ntracer
    mass = S.mass()
    fp = native.TracerFP(cfg, path="fused")
    o = pyoracle.Oracle(cfg)
    try:
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        fp.set_state(crp, cre, mass=mass)
        q = np.zeros_like(crp)

        class OracleFP:
            state = [crp.copy(), cre.copy()]

            def snapshot(self, bc, bn, z, zn, allow, dt, elapsed):
                o.snapshot(bc, bn, z, zn, allow, dt, elapsed, q, q, self.state[0], self.state[1], mass=mass)

        ref = []
        ofp = OracleFP()
        S.evolve(ofp, background=lambda i: pyoracle.background(S.raw_snapshot(i), PRM),
                 after=lambda i, el: ref.append(ofp.state[1].copy()))
        errs = []

        def check(i, el):
            _, g_cre = fp.get_state()
            errs.append(rel_err(g_cre, ref[i]))
            assert errs[-1] <= 1e-10, (i, errs[-1])

        end = S.evolve(fp, params=PRM, after=check)
        assert len(errs) == len(S) == 20 and end > 0.0
        assert np.any(fp.get_state()[1] != cre)
        print("worst over the written series", max(errs))
    finally:
        fp.close()


def test_series_emission_before_each_snapshot(tmp_path):
    """The series loop's before-hook sees the spectra a snapshot starts from,
    where the reference computes the emission: synchrotron and IC of the
    written series' tracers (the tracer_10k run's bands) from the hook at
    snapshot 0 equal those of the initial spectra computed on their own, and
    change once the spectra have evolved."""
    import series_io
    from croma_fp_b200 import histories
    series_io.write_series(str(tmp_path), nsnap=4)
    S = histories.SnapshotSeries(str(tmp_path), nb=128)
    cfg = config.tracer_10k(nb=128)
    emis = dict(nfreq=16, nu_min_s=5.5, nu_max_s=10.5, ntheta_pitch=512, nlogb=512, logb_min=-6.0, logb_max=2.0,
                nbins_ic=16, nu_min_ic=13.0, nu_max_ic=28.0)
    n = S.ntracer
    fp, alone = native.TracerFP(cfg, path="fused"), native.TracerFP(cfg, path="fused")
    try:
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), n, cfg.species)
        for f in (fp, alone):
            f.set_state(crp, cre, mass=S.mass())
            f.emission_setup(**emis)
        seen = {}
        S.evolve(fp, stop=3, params=PRM, before=lambda i, bg: seen.__setitem__(i, fp.emission_run(bg, S.z[i],
                                                                                                     kinds=("syn", "ic"))))
        first = alone.emission_run(S.background(0, PRM), S.z[0], kinds=("syn", "ic"))
        for k in ("syn", "ic"):
            assert np.array_equal(seen[0][k], first[k]), k
            assert np.all(np.isfinite(seen[2][k])) and np.any(seen[2][k] != seen[0][k]), k
        assert np.all(seen[0]["syn"] >= 0.0) and np.any(seen[0]["syn"] > 0.0)
    finally:
        fp.close()
        alone.close()
