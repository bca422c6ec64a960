"""croma_b200_step_host -- the per-snapshot step through host memory that the
bench's e2e figure times -- against the same step made of its parts on a
second context: croma_b200_dsa_inject (host shock fields), croma_b200_emission_run
(host outputs) and croma_b200_snapshot, then croma_b200_get_state.  The
emissivities and the evolved spectra must agree bit for bit (same kernels, same
inputs), over several consecutive steps, with both evolve forms; and the
result must match the oracle to the FP64 bar."""
import numpy as np
import pytest

from conftest import load_package
from golden_io import rel_err

load_package()
from croma_fp_b200 import config, native, synth  # noqa: E402

pytestmark = pytest.mark.gpu

EMIS = dict(nfreq=8, nu_min_s=7.0, nu_max_s=10.0, ntheta_pitch=32, nlogb=64, logb_min=-6.0, logb_max=2.0,
            nbins_ic=8, nu_min_ic=17.383, nu_max_ic=29.383, nbins_gamma=8, egamma_min=-6.0, egamma_max=6.0,
            nbins_nu=8, enu_min=-6.0, enu_max=6.0)


@pytest.mark.parametrize("path", ["fused", "plain"])
def test_step_host_equals_its_parts(path):
    cfg = config.config1(nb=128)
    nt, first, nsteps, seed = 96, 30, 3, 515
    w = synth.Workload(cfg, nt, 100, seed=seed)
    ctx = []
    for _ in range(2):
        fp = native.TracerFP(cfg, path=path)
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
        fp.set_state(crp, cre, mass=w.mass)
        fp.set_dsa(config.DsaParams())
        fp.emission_setup(**EMIS)
        ctx.append(fp)
    a, b = ctx
    import pyoracle
    o = pyoracle.Oracle(cfg)
    o_crp, o_cre = crp.copy(), cre.copy()
    qpi, qepri, dis = np.zeros_like(crp), np.zeros_like(cre), np.zeros(nt, np.uint8)
    try:
        for k in range(nsteps):
            isnap = first + k
            args = w.snapshot_args(isnap)
            sh = synth.shocks(args[0], isnap, seed, fraction=0.2)
            outs = {"syn": np.empty((nt, 8)), "ic": np.empty((nt, 8)), "gamma": np.empty((nt, 8)),
                    "nu": np.empty((nt, 8)), "crp": np.empty((nt, 128)), "cre": np.empty((nt, 128))}
            a.step_host(*args, shocks=sh, dsa_mode="tracer_state", outputs=outs)
            b.dsa_inject(sh, 1.0, args[5], "tracer_state")
            eps = b.emission_run(args[0], args[2])
            b.snapshot(*args, sync=True)
            g_crp, g_cre = b.get_state()
            for kk in ("syn", "ic", "gamma", "nu"):
                assert np.array_equal(outs[kk], eps[kk]), f"step {k}: {kk} differs"
            assert np.array_equal(outs["crp"], g_crp) and np.array_equal(outs["cre"], g_cre), f"step {k}"
            o.dsa_inject(config.DsaParams(), sh, w.mass, 1.0, args[5], 1, 0, o_crp, o_cre, qpi, qepri, dis)
            o.snapshot(*args, qpi, qepri, o_crp, o_cre, mass=w.mass, dis=dis)
            assert rel_err(outs["cre"], o_cre) <= 1e-10 and rel_err(outs["crp"], o_crp) <= 1e-10
    finally:
        a.close()
        b.close()


def test_step_host_spectra_only_and_no_shocks():
    """Outputs may be partial: no emission set up, no shock fields (no
    injection), only the electron spectra requested; the step equals
    snapshot + get_state on a second context."""
    cfg = config.config1(nb=128)
    nt, seed = 33, 616
    w = synth.Workload(cfg, nt, 100, seed=seed)
    ctx = []
    for _ in range(2):
        fp = native.TracerFP(cfg, path="fused")
        gp, ge = fp.grid(0), fp.grid(1)
        crp, cre = synth.initial_state((gp[0], gp[1]), (ge[0], ge[1]), nt, cfg.species)
        fp.set_state(crp, cre, mass=w.mass)
        ctx.append(fp)
    a, b = ctx
    try:
        for isnap in (40, 41):
            args = w.snapshot_args(isnap)
            out = {"cre": np.empty((nt, 128))}
            a.step_host(*args, outputs=out)
            b.snapshot(*args, sync=True)
            g_crp, g_cre = b.get_state()
            assert np.array_equal(out["cre"], g_cre)
        a_crp, a_cre = a.get_state()
        assert np.array_equal(a_crp, g_crp)
        with pytest.raises(native.CromaError):
            a.step_host(*args, outputs={"syn": np.empty((nt, 8))})   # emission never set up
    finally:
        a.close()
        b.close()
