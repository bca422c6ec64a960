"""ctypes mirror of the reference-compatible C ABI (include/fp_cuda_backend.h).

The structs reproduce the reference's field order (include/fp_cuda_backend.h
and include/fp_shared_core.h of kosukenishiwaki/croma-fp); ``CRspectrum`` is
sized by the bin count of the library loaded.  Used by the tests and by
Python callers that drive the drop-in entry points directly.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .native import load_library

_d, _i, _vp = C.c_double, C.c_int, C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_U8 = C.POINTER(C.c_ubyte)


def crspectrum_type(nb: int):
    class CRspectrum(C.Structure):
        _fields_ = [("p", _d * nb), ("dp", _d * nb), ("pp1", _d), ("pm1", _d), ("E", _d * nb),
                    ("N", _d * nb), ("N_pre", _d * nb), ("N_ave", _d * nb)]
    return CRspectrum


class FpCoeffBatchInput(C.Structure):
    _fields_ = [("ncell", _i), ("z", _d), ("dt_gyr", _d), ("epmax", _d),
                ("n_gas", _D), ("kbt", _D), ("b_field", _D), ("divv_gyr", _D), ("disable_adiabatic", _U8),
                ("l_turb_mpc", _D), ("dv_imc", _D), ("cs", _D), ("beta_pl", _D), ("tracer_mass_msun", _D),
                ("crp_state_cell_major", _D), ("cre_state_cell_major", _D),
                ("rad_ic_batch", _D), ("rad_ic_m1", _D), ("rad_ic_p1", _D),
                ("device_interp_background", _i), ("interp_alpha", _d),
                ("n_gas_next", _D), ("kbt_next", _D), ("b_field_next", _D), ("divv_gyr_next", _D),
                ("l_turb_mpc_next", _D), ("dv_imc_next", _D), ("cs_next", _D), ("beta_pl_next", _D),
                ("rad_ic_batch_next", _D), ("rad_ic_m1_next", _D), ("rad_ic_p1_next", _D)]


class FpSynchEmissionBatchInput(C.Structure):
    _fields_ = [("ncell", _i), ("nfreq", _i), ("nx_tab", _i), ("ntheta_pitch", _i), ("nlogb", _i),
                ("z", _d), ("xmin", _d), ("logb_min", _d), ("inv_dlogb", _d),
                ("fx_tab", _D), ("logfx_tab", _D), ("logx_tab", _D), ("logy", _vp),
                ("pitch_kernel_table", _D), ("b_dyn", _D), ("logb", _D), ("cre_batch", _D),
                ("gamma2e", _D), ("theta", _D), ("dtheta", _D), ("pitch_weight", _D), ("nus", _D)]


class FpHadronicEmissionBatchInput(C.Structure):
    """FpGammaEmissionBatchInput and FpNeutrinoEmissionBatchInput share this layout."""
    _fields_ = [("ncell", _i), ("nbins", _i), ("z", _d), ("e_min", _d), ("e_max", _d),
                ("n_gas", _D), ("crp_batch", _D), ("beta_p", _D), ("kernel_flat", _D)]


class FpIcEmissionBatchInput(C.Structure):
    _fields_ = [("ncell", _i), ("nbins", _i), ("z", _d), ("nu_min", _d), ("nu_max", _d),
                ("cre_batch", _D), ("fic_flat", _D)]


class FpChangCooperSolveBatchInput(C.Structure):
    _fields_ = [("nsys", _i), ("nrow", _i), ("dt", _d), ("a_batch", _D), ("b_batch", _D),
                ("c_batch", _D), ("source_batch", _D)]


class FpCudaOutputSchedule(C.Structure):
    _fields_ = [("emit_final_only", _i), ("emit_all_steps", _i), ("emit_stride", _i),
                ("physical_min", _i), ("physical_max", _i), ("selected_steps", _I),
                ("nselected_steps", _i)]


class FpCudaPipelineTimes(C.Structure):
    _fields_ = [(n, _d) for n in ("setup_ms", "h2d_ms", "device_interp_ms", "coeff_ms", "secondary_ms",
                                  "solve_ms", "diff_ms", "adv_ms", "synch_ms", "gamma_ms", "neutrino_ms",
                                  "d2h_ms", "other_ms", "total_ms")] + \
               [(n, _i) for n in ("emitted_synch", "emitted_gamma", "emitted_neutrino", "last_synch_step",
                                  "used_pcr_proton", "used_pcr_electron")]


def pipeline_input_type(nb: int):
    CR = crspectrum_type(nb)

    class FpCudaPipelineInput(C.Structure):
        _fields_ = [("ncell", _i), ("nstep", _i), ("fp_cadence_steps", _i), ("diff_cadence_steps", _i),
                    ("adv_cadence_steps", _i), ("use_windowed_reacc", _i), ("on_start_step", _i),
                    ("on_end_step", _i), ("nfreq", _i), ("nx_tab", _i),
                    ("dt", _d), ("epmax", _d), ("xmin", _d), ("psi_value", _d), ("mach_limit_value", _d),
                    ("transport_mode", _i),
                    ("crp_grid", C.POINTER(CR)), ("cre_grid", C.POINTER(CR)),
                    ("coeff_in", C.POINTER(FpCoeffBatchInput)), ("synch_in", _vp), ("gamma_in", _vp),
                    ("neutrino_in", _vp),
                    ("qpi_batch", _D), ("qepri_batch", _D), ("beta_p", _D), ("crp_init", _D), ("cre_init", _D),
                    ("crp_state_out", _D), ("cre_state_out", _D), ("eps_syn_out", _D), ("eps_gamma_out", _D),
                    ("eps_nu_out", _D), ("rank_state_indices", _I), ("gather_rank_state", _i),
                    ("scatter_rank_state", _i), ("workspace", _vp)]
    return CR, FpCudaPipelineInput


def dptr(a):
    return None if a is None else a.ctypes.data_as(_D)


def iptr(a):
    return None if a is None else a.ctypes.data_as(_I)


def u8ptr(a):
    return None if a is None else a.ctypes.data_as(_U8)


class RefAbi:
    """The fp_cuda_backend.h entry points of libcroma_b200_np<nb>.so."""

    def __init__(self, nb: int):
        self.nb = nb
        L = load_library(nb)
        self.lib = L
        self.CRspectrum, self.PipelineInput = pipeline_input_type(nb)
        L.cuda_pipeline_workspace_create.restype = _vp
        L.cuda_pipeline_workspace_destroy.argtypes = [_vp]
        L.cuda_rank_state_upload.argtypes = [_vp, _i, _D, _D, _D, _D, _D]
        L.cuda_rank_state_download.argtypes = [_vp, _i, _D, _D, _D]
        L.run_tracer_pipeline.argtypes = [C.POINTER(self.PipelineInput), C.POINTER(FpCudaOutputSchedule),
                                          _D, _D, _D, _D, _D, C.POINTER(FpCudaPipelineTimes)]
        L.run_pipeline_cuda.argtypes = L.run_tracer_pipeline.argtypes
        L.solve_cc_cuda_batch.argtypes = [C.POINTER(FpChangCooperSolveBatchInput), _D, _D, _D, _I]
        L.prepare_gamma_emission_cuda_batch.argtypes = [C.POINTER(FpHadronicEmissionBatchInput),
                                                        C.POINTER(self.CRspectrum), _D, _D]
        L.prepare_neutrino_emission_cuda_batch.argtypes = L.prepare_gamma_emission_cuda_batch.argtypes
        L.prepare_synch_emission_cuda_batch.argtypes = [C.POINTER(FpSynchEmissionBatchInput),
                                                        C.POINTER(self.CRspectrum), _D, _D]
        L.prepare_synch_pitch_kernel_table_cuda.argtypes = [C.POINTER(FpSynchEmissionBatchInput), _D, _D]
        L.cuda_get_current_device_id.argtypes = [C.c_char_p, _i]
        L.cuda_bind_local_rank.argtypes = [_i, _I]
        L.cuda_get_binding_state.argtypes = [_I, _I]
        L.fp_cuda_tridiag_solver_name.restype = C.c_char_p
        L.croma_b200_set_model.argtypes = [_i, _i, _d, _d]
        L.croma_b200_last_error.restype = C.c_char_p

    def error(self) -> str:
        return self.lib.croma_b200_last_error().decode()

    def kernel_table(self, fn: str, p, nbins: int, lo: float, hi: float, z: float = 0.0):
        """A device-built emission kernel table through its reference-form
        entry point (prepare_gamma_kernel_flat_cuda,
        prepare_neutrino_kernel_flat_cuda, prepare_ic_kernel_flat_cuda) for
        the momentum grid p: [nbins][nb]."""
        f = getattr(self.lib, fn)
        args = [C.POINTER(self.CRspectrum), _i, _d, _d] + ([_d] if fn == "prepare_ic_kernel_flat_cuda" else []) + [_D]
        f.argtypes = args
        zero = np.zeros(self.nb)
        g = self.grid(p, zero, zero, 0.0, 0.0)
        out = np.empty((nbins, self.nb))
        extra = [z] if fn == "prepare_ic_kernel_flat_cuda" else []
        if f(C.byref(g), nbins, lo, hi, *extra, dptr(out)) != 0:
            raise RuntimeError(self.error())
        return out

    def grid(self, p, dp, E, pm1, pp1):
        g = self.CRspectrum()
        g.p[:] = list(p)
        g.dp[:] = list(dp)
        g.E[:] = list(E)
        g.pm1 = pm1
        g.pp1 = pp1
        return g
