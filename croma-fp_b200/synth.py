"""Seeded synthetic tracer histories.

The reference reads tracer histories from HDF5 files or fills a seed-free
analytic "mock MHD" history (src/tracer_fp_debug.c:34-116).  The workloads
here instead draw, once per tracer and per snapshot, from the distributions
of the benchmark configurations:

* n_gas   log-uniform in [1e-5, 1e-2] cm^-3
* T       log-uniform in [1e6, 1e8] K
* |B|     log-uniform in [0.01, 10] muG (random direction; the magnitude is
          what the update uses)
* div v   normal, mean 0, sigma 1e-17 s^-1, converted to Gyr^-1
* |curl v| log-uniform in [1e-18, 1e-16] s^-1

and convert them to the update's inputs exactly as the reference's
background preparation does (prepare_background_cell,
src/fp_shared_core.c:866-932, with bfield_mode = max, mu_mol = 0.59,
eta_B = 0.05, L_turb_target = 150 kpc): kbt, the dynamo / simulation field
maximum, dv = |curl v| * l_turb limited to mach_limit * c_s, c_s, beta_pl.

Random numbers come from numpy's Philox counter generator keyed by
(seed, snapshot), so every snapshot can be regenerated independently and
identically on any machine.  Snapshots are evenly spaced in redshift; the
time step between them is the flat-LCDM cosmic-time difference
(H0 = 70 km/s/Mpc, Omega_m = 0.3) computed by Gauss-Legendre quadrature.
"""
from __future__ import annotations

import numpy as np

# Constants of src/CONSTANTS.c and src/params.c used by background prep.
C_LIGHT = 2.999e10
KB_EV = 8.62e-5
EV = 1.6e-12
GYR = 3.1536e16
MPC = 3.0857e24
KPC = 3.0857e21
MU_MOL = 0.59
ETA_B = 0.05
M_SUN = 1.99e33

BG_FIELDS = ("n_gas", "kbt", "b_field", "divv_gyr", "l_turb_mpc", "dv_imc", "cs", "beta_pl")
NBG = len(BG_FIELDS)


def _rng(seed: int, snapshot: int) -> np.random.Generator:
    ss = np.random.SeedSequence([int(seed) & 0xFFFFFFFF, int(snapshot) & 0xFFFFFFFF, 0xC20A])
    return np.random.Generator(np.random.Philox(ss))


def _log_uniform(rng, lo, hi, n):
    return 10.0 ** rng.uniform(np.log10(lo), np.log10(hi), n)


def background(ntracer: int, snapshot: int, seed: int, mach_limit: float = 0.5) -> np.ndarray:
    """Field-major background block [8][ntracer] (order BG_FIELDS)."""
    rng = _rng(seed, snapshot)
    n_gas = _log_uniform(rng, 1e-5, 1e-2, ntracer)
    temp = _log_uniform(rng, 1e6, 1e8, ntracer)
    b_mag_ug = _log_uniform(rng, 0.01, 10.0, ntracer)
    _direction = rng.normal(size=(3, ntracer))          # isotropic; magnitude is used
    div_v = rng.normal(0.0, 1e-17, ntracer)
    curl_v = _log_uniform(rng, 1e-18, 1e-16, ntracer)

    temp = np.maximum(temp, 1.0e4)
    l_turb_cm = 150.0 * KPC
    cs = np.sqrt(5.0 / 3.0 * KB_EV * temp / (MU_MOL * 0.938 * 1.0e9)) * C_LIGHT
    dv = curl_v * l_turb_cm
    if mach_limit > 0.0:
        dv = np.where((cs > 0.0) & (dv / cs > mach_limit), mach_limit * cs, dv)
    density = n_gas * (1.6e-24 * MU_MOL)
    b_sim = b_mag_ug * 1.0e-6
    b_dyn = np.sqrt(4.0 * np.pi * ETA_B * density * dv * dv)
    b_eff = np.maximum(b_dyn, b_sim)
    beta_pl = np.where(b_eff > 0.0, n_gas * KB_EV * temp * EV / (b_eff * b_eff / (8.0 * np.pi)), 1.0e10)

    out = np.empty((NBG, ntracer), dtype=np.float64)
    out[0] = n_gas
    out[1] = KB_EV * temp * 1.0e-9
    out[2] = b_eff
    out[3] = div_v * GYR
    out[4] = l_turb_cm / MPC
    out[5] = dv
    out[6] = cs
    out[7] = beta_pl
    return out


def shocks(bg: np.ndarray, snapshot: int, seed: int, fraction: float = 0.05,
           merged: bool = False) -> dict:
    """Seeded shock fields for one snapshot: each tracer is shocked with
    probability `fraction` (Bernoulli per tracer-snapshot) with Mach number
    U[2, 5]; the upstream temperature and density are the tracer's own
    background (kbt, n_gas), density_unit = 1.  `merged` gives the merged-DSA
    form (trigger, Mach, pre-shock density, kinetic energy flux 0.5 rho u^3 at
    u = M cs) instead of (mach, prestemp, presden, side code)."""
    n = bg.shape[1]
    rng = _rng(seed ^ 0x5A5A5A5A, snapshot)
    hit = rng.uniform(size=n) < fraction
    mach = np.where(hit, rng.uniform(2.0, 5.0, n), 0.0)
    temp = bg[1] * 1.0e9 / KB_EV
    rho = bg[0] * (1.6e-24 * MU_MOL)
    if merged:
        u = mach * bg[6]
        return {"has_dsa": 1, "dsa_trigger": hit.astype(np.float64), "dsa_mach": mach,
                "dsa_pre_density": rho, "dsa_flux_cgs": 0.5 * rho * u * u * u,
                "shock_side_code": np.where(hit, 1.0, 99.0)}
    return {"has_dsa": 0, "mach": mach, "prestemp": temp, "presden": rho,
            "shock_side_code": np.where(hit, 1.0, 99.0)}


def _cosmic_time_gyr(z: float, h0: float = 70.0, om: float = 0.3) -> float:
    """Age of a flat LCDM universe at redshift z, in Gyr."""
    ol = 1.0 - om
    h0_s = h0 * 1.0e5 / MPC
    x, w = np.polynomial.legendre.leggauss(200)
    # t(z) = int_z^inf dz' / ((1+z') H(z')); substitute a = 1/(1+z')
    a_hi = 1.0 / (1.0 + z)
    a = 0.5 * a_hi * (x + 1.0)
    integrand = 1.0 / (a * np.sqrt(om / a**3 + ol)) / a
    val = 0.5 * a_hi * np.sum(w * integrand * a)
    return val / h0_s / GYR


def timeline(nsnap: int, z_start: float = 1.0, z_end: float = 0.0):
    """Redshifts evenly spaced from z_start to z_end and the cosmic-time step
    (Gyr) from each snapshot to the next (the last repeats the previous)."""
    z = np.linspace(z_start, z_end, nsnap)
    t = np.array([_cosmic_time_gyr(float(zz)) for zz in z])
    dt = np.empty(nsnap)
    if nsnap > 1:
        dt[:-1] = np.diff(t)
        dt[-1] = dt[-2]
    else:
        dt[0] = t[0] * 0.01
    return z, dt


def initial_state(grid_p: np.ndarray, grid_e: np.ndarray, ntracer: int, species: str,
                  delta: float = 2.5, mass_msun: float = 1.0e7, phi: float = 1.0e-6):
    """Cell-major initial spectra (crp [ntracer][nb], cre [ntracer][nb]).

    Power law N(p) ~ p^-delta with the reference's template cut-offs
    (initial_cr_*_template, src/tracer_fp_cr_source.c:6-14: peinjmin = 10,
    pinjmin = 1, pinjmax = 1e6) and the number normalisation of
    CRe_Norm / CRp_Norm (:41-72) for a tracer of mass_msun.
    grid_* are (p, dp) pairs.
    """
    p_p, dp_p = grid_p
    p_e, dp_e = grid_e
    te = p_e ** (-delta) * np.exp(-10.0 / p_e)
    tp = p_p ** (-delta) * np.exp(-1.0 / p_p) * np.exp(-p_p / 1.0e6)
    n_th = 0.52 * mass_msun * M_SUN / (MU_MOL * 1.6e-24)
    num_e = np.sum(np.where(p_e > 10.0, te * dp_e, 0.0))
    num_p = np.sum(np.where(p_p > 1.0, tp * dp_p, 0.0))
    ne = phi / (num_e / n_th) * te
    npp = phi / (num_p / n_th) * tp
    cre = np.zeros((ntracer, p_e.size))
    crp = np.zeros((ntracer, p_p.size))
    if species in ("electron_only", "electron_proton"):
        cre[:] = ne
    if species in ("proton_only", "electron_proton"):
        crp[:] = npp
    return crp, cre


class Workload:
    """A seeded synthetic run: backgrounds per snapshot, timeline, initial
    spectra and (zero) sources for ntracer tracers."""

    def __init__(self, cfg, ntracer: int, nsnap: int, seed: int = 1234):
        self.cfg = cfg
        self.ntracer = int(ntracer)
        self.nsnap = int(nsnap)
        self.seed = int(seed)
        self.z, self.dt = timeline(self.nsnap)
        self.elapsed = np.concatenate([[0.0], np.cumsum(self.dt)[:-1]])
        self.mass = np.full(self.ntracer, 1.0e7)

    def background(self, isnap: int) -> np.ndarray:
        return background(self.ntracer, isnap, self.seed, self.cfg.mach_limit)

    def snapshot_args(self, isnap: int):
        """(bg_curr, bg_next, z_curr, z_next, allow_interp, dt, elapsed)."""
        cur = self.background(isnap)
        allow = isnap + 1 < self.nsnap
        nxt = self.background(isnap + 1) if allow else cur
        z_next = self.z[isnap + 1] if allow else self.z[isnap]
        return cur, nxt, float(self.z[isnap]), float(z_next), bool(allow), float(self.dt[isnap]), float(self.elapsed[isnap])
