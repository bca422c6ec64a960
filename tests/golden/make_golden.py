"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference ships no tests, golden vectors or fixtures for this path, so
its own CPU implementation -- compiled from its sources by
`make -C oracle ref` into oracle/_ref/libcroma_ref_np<N>.so -- is run here on
seeded synthetic tracers, and its outputs are stored with their inputs.

Run from the repository root (needs the reference tree at build time; its
location is CROMA_REFERENCE_ROOT):

    make -C oracle ref && python tests/golden/make_golden.py

Each case file golden_<name>.npz holds the run configuration, the inputs
(backgrounds per snapshot, timeline, initial spectra) and the reference's
outputs after every snapshot (nsub, n_on, bucket ids, spectra), plus the
IC-cooling rows and the one-time grid tables.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from conftest import load_package  # noqa: E402

load_package()
from croma_fp_b200 import config, synth  # noqa: E402
import pyoracle  # noqa: E402

CASES = {
    # name: (config factory kwargs, ntracer, first snapshot, nsnap run, seed, timeline length)
    "c0_direct": (("config0", dict(nsub_max=500)), 16, 0, 3, 101, 100),
    "c0_last": (("config0", dict(nsub_max=500)), 8, 98, 2, 102, 100),
    "c0_nocap": (("config0", dict(nsub_max=0)), 3, 97, 1, 103, 100),
    "c1_asa256": (("config1", dict()), 6, 10, 2, 104, 100),
    "c1_asa128": (("config1", dict(nb=128)), 8, 0, 2, 105, 100),
    "c2_ttd": (("config2", dict()), 8, 20, 2, 106, 100),
    "c2_ttd_spect_window": (("config2", dict(ttd_tacc_model=0, reacc_window_mode=1, f_eddy=0.001)),
                            8, 40, 2, 107, 100),
    "c0_narrow": (("config0", dict(pemin=1.0, pemax=3.0, nsub_max=500)), 32, 30, 3, 109, 100),
    "c1_narrow_window": (("config1", dict(nb=128, pmin=0.0, pmax=3.0, pemin=1.0, pemax=3.0,
                                          reacc_window_mode=1, f_eddy=0.002)), 32, 50, 2, 110, 100),
    "c4_asa512": (("config4", dict()), 3, 60, 1, 108, 100),
    # eta cap binding for most tracers, with protons and electrons evolving
    "c1_etacap": (("config1", dict(nb=128, eta_dpp_cap=1.0)), 8, 30, 2, 111, 100),
}


def make_case(name, spec):
    (factory, kw), nt, isnap0, nrun, seed, nsnap = spec
    cfg = getattr(config, factory)(**kw)
    ref = pyoracle.ReferenceCPU(cfg)
    w = synth.Workload(cfg, nt, nsnap, seed=seed)
    gp, ge = ref.grid(0), ref.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    qpi = np.zeros_like(crp)
    qepri = np.zeros_like(cre)
    out = dict(config=json.dumps(cfg.__dict__), ntracer=nt, isnap0=isnap0, nrun=nrun, seed=seed,
               nsnap=nsnap, z=w.z, dt=w.dt, elapsed=w.elapsed, mass=w.mass,
               crp0=crp.copy(), cre0=cre.copy())
    bgs = []
    for k in range(nrun + 1):
        bgs.append(w.background(isnap0 + k) if isnap0 + k < nsnap else w.background(isnap0 + k - 1))
    out["bg"] = np.stack(bgs)
    for k in range(nrun):
        isnap = isnap0 + k
        allow = isnap + 1 < nsnap
        cur = out["bg"][k]
        nxt = out["bg"][k + 1] if allow else cur
        z_next = w.z[isnap + 1] if allow else w.z[isnap]
        ic = ref.ic_row(w.z[isnap])
        out[f"ic_row_{k}"] = np.concatenate([ic[0], [ic[1], ic[2]]])
        nsub, non, bid, nb = ref.snapshot(cur, nxt, float(w.z[isnap]), float(z_next), allow,
                                          float(w.dt[isnap]), float(w.elapsed[isnap]), qpi, qepri,
                                          crp, cre, mass=w.mass)
        out[f"nsub_{k}"] = nsub
        out[f"non_{k}"] = non
        out[f"bucket_ids_{k}"] = bid
        out[f"crp_{k}"] = crp.copy()
        out[f"cre_{k}"] = cre.copy()
    out["grid_p"] = np.concatenate([gp[0], gp[1], gp[2], [gp[3], gp[4]]])
    out["grid_e"] = np.concatenate([ge[0], ge[1], ge[2], [ge[3], ge[4]]])
    s, g, j = ref.pp_cache()
    out["sigma_pp"], out["sigmoid_pp"], out["j_pp"] = s, g, j
    fqe, npmin = ref.secondary_kernel()
    out["np_min_qe"] = npmin
    if cfg.nb == 128:
        out["fqe"] = fqe
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)
    print(name, "nsub range", [(int(out[f"nsub_{k}"].min()), int(out[f"nsub_{k}"].max())) for k in range(nrun)])


# DSA injection cases: (nb, ntracer, snapshot, seed, shocked fraction, state scale)
DSA_CASES = {
    "dsa_128": (128, 32, 20, 301, 0.4, 1.0e3),
    "dsa_256": (256, 24, 40, 302, 0.4, 1.0e3),
}


def make_dsa_case(name, spec):
    """Every (shock form, injection mode, reacceleration mode) combination of
    the reference's tracer_fp_apply_dsa_tracer_injection_snapshot on one set
    of tracers; drury83 runs with its eta cap on."""
    nb, nt, isnap, seed, frac, scale = spec
    cfg = config.config1(nb=nb)
    ref = pyoracle.ReferenceCPU(cfg)
    w = synth.Workload(cfg, nt, 100, seed=seed)
    bg = w.background(isnap)
    gp, ge = ref.grid(0), ref.grid(1)
    crp0, cre0 = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
    crp0 *= scale
    cre0 *= scale
    out = dict(nb=nb, ntracer=nt, isnap=isnap, seed=seed, fraction=frac, dt=float(w.dt[isnap]),
               mass=w.mass, bg=bg, crp0=crp0, cre0=cre0)
    for merged in (0, 1):
        sh = synth.shocks(bg, isnap, seed, fraction=frac, merged=bool(merged))
        for k, v in sh.items():
            out[f"shock{merged}_{k}"] = np.asarray(v, dtype=np.float64)
        for mode in (1, 2):
            for reacc in (0, 1, 2):
                prm = config.DsaParams(reacc_eta_cap=0.05 if reacc == 2 else 0.0)
                crp, cre = crp0.copy(), cre0.copy()
                qpi, qe = np.zeros_like(crp), np.zeros_like(cre)
                dis = np.zeros(nt, np.uint8)
                n = ref.dsa_inject(prm, sh, w.mass, 1.0, float(w.dt[isnap]), mode, reacc, crp, cre,
                                   qpi, qe, dis)
                tag = f"m{merged}_mode{mode}_r{reacc}"
                out[f"{tag}_crp"], out[f"{tag}_cre"] = crp, cre
                out[f"{tag}_qpi"], out[f"{tag}_qepri"] = qpi, qe
                out[f"{tag}_dis"], out[f"{tag}_ninj"] = dis, np.int32(n)
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)
    print(name, "written")


def make_ic_emission(name="emission_ic"):
    """IC emissivities of the reference (prepare_ic_kernel_flat +
    prepare_ic_emission_batch) for 128- and 256-bin electron spectra."""
    out = {}
    for nb in (128, 256):
        cfg = config.config1(nb=nb)
        ref = pyoracle.ReferenceCPU(cfg)
        w = synth.Workload(cfg, 12, 100, seed=404)
        gp, ge = ref.grid(0), ref.grid(1)
        _, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), 12, cfg.species)
        cre = cre * np.random.default_rng(nb).uniform(0.5, 2.0, (12, 1))
        fic, eps = ref.ic_emission(cre, 20, 0.3, 14.0, 26.0)
        out[f"nb{nb}_cre"], out[f"nb{nb}_fic"], out[f"nb{nb}_eps"] = cre, fic, eps
        out[f"nb{nb}_dp"] = ge[1]
    out["z"], out["nu_min"], out["nu_max"], out["nbins"] = 0.3, 14.0, 26.0, 20
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)
    print(name, "written")


def synch_inputs(ge_p, nfreq, ntheta, nu_min=5.5, nu_max=10.5):
    """Synchrotron tables built the way tracer_fp_synch_data_init_tables
    (src/tracer_fp_synch.c:87-121) builds them: logx grid [-25, 2.5) in 2750
    cells, pitch angles (k + 1/2) pi / ntheta with sin^2 weights, log-spaced
    frequencies, logy = log10(nu / (1e-6 nu_crit)) with
    nu_crit = (1 + p^2) 4.194284e6 sin(theta) (src/Synchrotron.c:9-51).  The
    F(x) values are a smooth positive stand-in, x^(1/3) e^(-x) scaled, not
    the synchrotron function itself: what is checked is the lookup and the
    integration, which do not depend on the values."""
    nx, xmin, xmax = 2750, -25.0, 2.5
    dx = (xmax - xmin) / nx
    logx = xmin + dx * np.arange(nx)
    x = 10.0 ** logx
    fx = 2.15 * x ** (1.0 / 3.0) * np.exp(-x) + 1e-300
    logfx = np.log10(fx)
    fx = 10.0 ** logfx
    theta = (np.arange(ntheta) + 0.5) * np.pi / ntheta
    w = np.sin(theta) * np.sin(theta) * (np.pi / ntheta)
    dnu = (nu_max - nu_min) / nfreq
    nus = 10.0 ** (nu_min + dnu * np.arange(nfreq))
    nu_crit = (1.0 + ge_p[:, None] ** 2) * 4.194284e6 * np.sin(theta)[None, :]
    logy = np.log10(nus[:, None, None] / (1.0e-6 * nu_crit[None, :, :]))
    return dict(logx=logx, logfx=logfx, fx=fx, xmin=xmin, w=w, logy=np.ascontiguousarray(logy))


def make_synch_emission(name="emission_synch"):
    """The reference's pitch-kernel table and both branches of its
    synchrotron emissivity (with and without the table) on 128-bin spectra,
    some cut off at high momenta so the stop rule at N[je+1] <= 0 acts."""
    nb, ncell, nfreq, ntheta, nlogb = 128, 10, 6, 16, 24
    cfg = config.config1(nb=nb)
    ref = pyoracle.ReferenceCPU(cfg)
    gp, ge = ref.grid(0), ref.grid(1)
    _, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), ncell, cfg.species)
    rng = np.random.default_rng(77)
    cre = cre * rng.uniform(0.5, 2.0, (ncell, 1))
    for i, cut in enumerate((112, 121, 3, 127)):
        cre[i, cut:] = 0.0
    b_dyn = 10.0 ** rng.uniform(-7.5, -5.0, ncell)
    logb = np.log10(b_dyn)
    t = synch_inputs(ge[0], nfreq, ntheta)
    logb_min, logb_max = -8.0, -4.0
    inv_dlogb = (nlogb - 1) / (logb_max - logb_min)
    table = ref.synch_pitch_table(t["logy"], t["w"], logb_min, inv_dlogb, nlogb, t["xmin"], t["logx"],
                                  t["logfx"], t["fx"])
    eps_table = ref.synch_emission(cre, b_dyn, logb, t["logy"], t["w"], t["xmin"], t["logx"], t["logfx"],
                                   t["fx"], table=table, logb_min=logb_min, inv_dlogb=inv_dlogb)
    eps_theta = ref.synch_emission(cre, b_dyn, logb, t["logy"], t["w"], t["xmin"], t["logx"], t["logfx"],
                                   t["fx"])
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), nb=nb, cre=cre, dp=ge[1], b_dyn=b_dyn,
                        logb=logb, logb_min=logb_min, inv_dlogb=inv_dlogb, nlogb=nlogb, table=table,
                        eps_table=eps_table, eps_theta=eps_theta, **t)
    print(name, "written")


# Emission tables of the config-4 kind at a small size: band grids as
# config 4 states them (1 keV .. 1 PeV for gamma / neutrino in log10 GeV, the
# same photon energies for IC in log10 Hz, synchrotron 10 MHz .. 10 GHz).
EMIS_TABLES = dict(nb=128, nbins=16, egamma=(-6.0, 6.0), enu=(-6.0, 6.0),
                   nu_ic=(17.383, 29.383), z_ic=0.5, nfreq=8, nu_s=(7.0, 10.0), ntheta=32, nlogb=512,
                   logb=(-6.0, 2.0), plane_stride=16, ncell=12)


def make_emission_tables(name="emission_tables"):
    """The reference's own kernel tables (prepare_gamma/neutrino/ic_kernel_flat),
    synchrotron tables (tracer_fp_synch_data_init_tables with the checker's
    F(x) in place of GSL's, the pitch-kernel table of
    tracer_fp_refresh_synch_kernel_table over the default log-B range) and
    emissivities (prepare_*_emission_cell_major) on 128-bin e+p spectra,
    some electron spectra cut off so that the synchrotron stop rule acts.
    Every plane_stride-th log-B plane of the pitch table is kept."""
    e = EMIS_TABLES
    nb, nbins = e["nb"], e["nbins"]
    cfg = config.config1(nb=nb)
    ref = pyoracle.ReferenceCPU(cfg)
    gp, ge = ref.grid(0), ref.grid(1)
    crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), e["ncell"], cfg.species)
    rng = np.random.default_rng(4401)
    crp = crp * rng.uniform(0.5, 2.0, (e["ncell"], 1))
    cre = cre * rng.uniform(0.5, 2.0, (e["ncell"], 1))
    for i, cut in enumerate((100, 121, 3, 127)):
        cre[i, cut:] = 0.0
    bg = synth.background(e["ncell"], 7, 4402)
    n_gas, b_field = bg[0].copy(), bg[2].copy()
    b_field[5] = 0.0   # a non-positive field takes the 1e-30 G floor
    out = dict(nb=nb, cre=cre, crp=crp, n_gas=n_gas, b_field=b_field, dp_e=ge[1], dp_p=gp[1], p_e=ge[0],
               p_p=gp[0])
    out["fga"] = ref.kernel_table("gamma", nbins, *e["egamma"])
    out["fnu"] = ref.kernel_table("nu", nbins, *e["enu"])
    out["fic"] = ref.kernel_table("ic", nbins, *e["nu_ic"], z=e["z_ic"])
    out["eps_gamma"] = ref.hadronic_emission("gamma", crp, n_gas, out["fga"], *e["egamma"])
    out["eps_nu"] = ref.hadronic_emission("nu", crp, n_gas, out["fnu"], *e["enu"])
    fic2, out["eps_ic"] = ref.ic_emission(cre, nbins, e["z_ic"], *e["nu_ic"])
    assert np.array_equal(fic2, out["fic"])
    r = ref.synch_run(e["nfreq"], *e["nu_s"], e["ntheta"], e["nlogb"], *e["logb"], b_field=b_field, cre=cre)
    for k in ("logx", "logfx", "fx", "theta", "w", "nus", "logy"):
        out["syn_" + k] = r[k]
    out["syn_table_planes"] = r["table"][::e["plane_stride"]].copy()
    out["eps_syn"] = r["eps"]
    out["params"] = json.dumps(e)
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)
    print(name, "written")


HISTORY_SNAPS = (0, 1, 2, 3, 97, 98, 99)   # of the 100-file series: its start and its end
LONG_SNAPS = 20


def make_histories(name="histories"):
    """Real tracer histories: the reference's tracer_10k snapshot series
    (dump0025 .. dump0124) read by the library's HDF5 reader, every 39th of
    the 10,000 tracers (256), snapshots HISTORY_SNAPS of the series.  Stored:
    the raw fields each snapshot's background reads (with the previous and
    next snapshots' curl_v), the unit factors, redshifts and run-loop flags,
    the timeline (z, z_next, dt), the masses, and the reference's own
    prepare_background_cell outputs (oracle/_ref) for the default run
    parameters; and the raw fields of the first 64 of those tracers over the
    first LONG_SNAPS snapshots (long<k>_<field>), with every snapshot's unit
    factors."""
    from croma_fp_b200 import histories
    refroot = os.environ.get("CROMA_REFERENCE_ROOT", "/root/reference")
    S = histories.SnapshotSeries(os.path.join(refroot, "tracer_10k"))
    idx = np.arange(0, S.ntracer, 39)[:256]
    out = {"tracers": idx, "mass": S.mass()[idx], "z": S.z, "z_next": S.z_next, "dt": S.dt,
           "snaps": np.array(HISTORY_SNAPS), "params": json.dumps(histories.DEFAULT_BACKGROUND)}
    for i in HISTORY_SNAPS:
        raw = S.raw_snapshot(i)
        sel = {k: (np.ascontiguousarray(v[idx]) if isinstance(v, np.ndarray) else v) for k, v in raw.items()}
        for k, v in sel.items():
            out[f"s{i}_{k}"] = np.asarray(v)
        out[f"s{i}_bg_ref"] = pyoracle.reference_background(sel, histories.DEFAULT_BACKGROUND)
    # the first 64 of those tracers over the first LONG_SNAPS snapshots, raw
    long_idx = idx[:64]
    out["c_dens"], out["c_mag"] = S.c_dens, S.c_mag
    for k in range(LONG_SNAPS):
        for f, v in S.raw(k).items():
            out[f"long{k}_{f}"] = np.ascontiguousarray(v[long_idx])
    out["long_mass"] = S.mass()[long_idx]
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)
    print(name, "written")


if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES) + list(DSA_CASES) + ["emission_ic", "emission_synch", "emission_tables",
                                                              "histories"]
    for n in names:
        if n == "histories":
            make_histories(n)
        elif n in DSA_CASES:
            make_dsa_case(n, DSA_CASES[n])
        elif n == "emission_ic":
            make_ic_emission(n)
        elif n == "emission_synch":
            make_synch_emission(n)
        elif n == "emission_tables":
            make_emission_tables(n)
        else:
            make_case(n, CASES[n])
