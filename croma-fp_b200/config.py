"""Run configuration for the tracer Fokker-Planck update.

Field names and defaults mirror the reference's parameter globals
(src/params.c:78-115 in kosukenishiwaki/croma-fp): the momentum grid
bounds pmin/pmax/pemin/pemax (log10 of p/(m c)), Dpp_mode, t_acc_direct_gyr,
mach_limit, psi, eta_dpp_cap, tracer_nsub_safety, tracer_nsub_max,
coeff_interp_min_steps, coeff_interp_max_segments, reacc_window_mode,
f_eddy, t_off_gyr, t_acc_off_gyr and ttd_tacc_model.  The bin counts
np == npe == nb are compile-time macros there (include/params.h:22-27) and a
field here.
"""
from __future__ import annotations

import dataclasses

DPP_MODELS = {"asa": 1, "ttd": 2, "off": 3, "direct_tacc": 4}
SPECIES = ("electron_only", "proton_only", "electron_proton")


@dataclasses.dataclass
class RunConfig:
    nb: int = 128
    species: str = "electron_only"
    pmin: float = -2.0
    pmax: float = 6.0
    pemin: float = -1.0
    pemax: float = 6.0
    dpp_mode: str = "direct_tacc"
    ttd_tacc_model: int = 1            # 0 spectral, 1 brunetti16 (params.c:74-75)
    t_acc_direct_gyr: float = 0.3
    mach_limit: float = 0.5
    psi: float = 0.5
    eta_dpp_cap: float = 0.0
    nsub_safety: float = 0.25
    nsub_max: int = 500
    coeff_interp_min_steps: int = 4
    coeff_interp_max_segments: int = 16
    reacc_window_mode: int = 0         # 0 always on, 1 centred window
    f_eddy: float = 2.0
    t_off_gyr: float = 0.0
    t_acc_off_gyr: float = 3.0

    def dpp_model_id(self) -> int:
        return DPP_MODELS[self.dpp_mode]

    def species_mask(self) -> int:
        """bit 0: protons evolve, bit 1: electrons evolve.  `species` names the
        seed spectra (seed_cr_species, src/params.c:69); the reference evolves
        both species whatever the seed, so the mask leaves out only a species
        that stays zero: protons of an electron-only seed.  A proton seed
        feeds secondary electrons, so both evolve."""
        return {"electron_only": 2, "proton_only": 3, "electron_proton": 3}[self.species]


def config0(**kw) -> RunConfig:
    """Plain FP64 electron_only workload: 128 bins, p_e in [1e-1, 1e6],
    direct t_acc = 0.3 Gyr."""
    base = dict(nb=128, species="electron_only", pemin=-1.0, pemax=6.0,
                dpp_mode="direct_tacc", t_acc_direct_gyr=0.3)
    base.update(kw)
    return RunConfig(**base)


def config1(**kw) -> RunConfig:
    """Batching workload: electron_proton, 256 bins per species, protons over
    p/(m_p c) in [1e-2, 1e6], ASA reacceleration, nsub capped at 500."""
    base = dict(nb=256, species="electron_proton", pmin=-2.0, pmax=6.0,
                pemin=-1.0, pemax=6.0, dpp_mode="asa", nsub_max=500)
    base.update(kw)
    return RunConfig(**base)


def config2(**kw) -> RunConfig:
    """Precision workload: electron_only, 128 bins, TTD reacceleration."""
    base = dict(nb=128, species="electron_only", pemin=-1.0, pemax=6.0,
                dpp_mode="ttd", nsub_max=500)
    base.update(kw)
    return RunConfig(**base)


def config4(**kw) -> RunConfig:
    """Full pipeline: electron_proton with pp secondaries, 512 bins, ASA."""
    base = dict(nb=512, species="electron_proton", pmin=-2.0, pmax=6.0,
                pemin=-1.0, pemax=6.0, dpp_mode="asa", nsub_max=500)
    base.update(kw)
    return RunConfig(**base)


def tracer_10k(**kw) -> RunConfig:
    """The reference's run of its real tracer histories (params_tracer_10k.txt
    in kosukenishiwaki/croma-fp): electron_only seeds, p_p in [1e-1, 1e8],
    p_e in [10^-0.5, 1e6], ASA reacceleration in a centred window, eta cap
    0.1, sub-step safety 0.5."""
    base = dict(nb=128, species="electron_only", pmin=-1.0, pmax=8.0, pemin=-0.5, pemax=6.0,
                dpp_mode="asa", reacc_window_mode=1, eta_dpp_cap=0.1, nsub_safety=0.5, mach_limit=0.5, psi=0.5,
                nsub_max=0)
    base.update(kw)
    return RunConfig(**base)


DSA_MODELS = ("KR07", "KR07r", "KR13", "KR13r", "CS14", "CS14r", "Ryu19", "Ryu19r")
DSA_MODE = {"off": 0, "tracer_state": 1, "tracer_source": 2}
DSA_REACC = {"off": 0, "positive_delta": 1, "drury83": 2}


@dataclasses.dataclass
class DsaParams:
    """DSA injection parameters, mirroring the reference's globals
    (src/params.c:96-113, mu_mol :127) and the DSA grid bounds of
    src/tracer_fp.c:841 (dsa_init_grid(..., -3.0, -3.0)).  Efficiency models
    are indices into DSA_MODELS (the DSAModelID order)."""
    eta_model_initial: int = 6        # Ryu19
    eta_model_reacc: int = 7          # Ryu19r
    chi_p: float = 3.5
    chi_e: float = 3.5
    k_ep: float = 1.0e-2
    pmax_p_mc: float = 1.0e6
    pmax_e_mc: float = 1.0e5
    min_mach: float = 1.5
    gamma_gas: float = 5.0 / 3.0
    xcr_pmin_pmc: float = 1.0
    reacc_eta_cap: float = 0.0
    mu_mol: float = 0.59
    pmin_dsa_p_log10: float = -3.0
    pmin_dsa_e_log10: float = -3.0
    inject_species: int = 0           # 0 both, 1 electrons, 2 protons

