"""ctypes binding of libcathode_b200.so (the C ABI of include/cathode_b200.h).

The binding is the only path from Python to the product: every call goes
through the shared library's extern "C" entry points.  There is no CPU
fallback; loading fails loudly when the library is missing or was built
without CUDA.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcathode_b200.so")

CTH_OK = 0
CTH_NOT_CONVERGED = 1
CTH_NONFINITE = 2
CTH_ERR_ARG = -1
CTH_ERR_CUDA = -2
CTH_ERR_ALLOC = -3
CTH_ERR_UNSUPPORTED = -4

CTH_PREC_FP64 = 0
CTH_PREC_MIXED = 1

# every symbol include/cathode_b200.h declares
EXPORTS = (
    "cth_version", "cth_last_error", "cth_grid_create", "cth_grid_destroy", "cth_grid_ld",
    "cth_grid_levels", "cth_grid_set_cycle", "cth_smg_solve", "cth_smg_solve_dev", "cth_smg_solve_guess_dev", "cth_sor_solve",
    "cth_sor_solve_dev", "cth_residual_dev", "cth_to_device_layout", "cth_from_device_layout",
    "cth_launch_count", "cth_profile", "cth_profile_read", "cth_residual_noalloc", "cth_grid_set_graphs", "cth_grid_set_tail", "cth_grid_set_reuse", "cth_grid_reuse_stats", "cth_grid_time_relax", "cth_grid_time_cycle",
    "cth_c5_solve", "cth_c5_solve_dev", "cth_mw_er_assemble_dev",
    "cth_mw3_create", "cth_mw3_destroy", "cth_mw3_ld", "cth_mw3_launch_count", "cth_mw3_assemble_dev",
    "cth_mw3_copy_planes", "cth_mw3_apply_dev", "cth_mw3_solve_dev", "cth_mw3_solve_guess_dev", "cth_mw3_set_graphs",
    "cth_mw3_create_blocks", "cth_mw3_set_boundary", "cth_mw3_assemble_explicit_dev", "cth_mw3_fill_ghosts", "cth_mw3_set_cycle", "cth_mw3_set_preconditioner", "cth_mw3_set_precision",
    "cth_fields_create", "cth_fields_destroy", "cth_fields_set_warm_start", "cth_fields_set_download_plan", "cth_fields_download_wait", "cth_fields_set_upload_plan", "cth_fields_upload_many",
    "cth_fields_download_many", "cth_field", "cth_field_upload", "cth_field_download",
    "cth_flags_upload", "cth_table_upload", "cth_update_transport_coef", "cth_solve_phi_pc",
    "cth_ghost_rules_upload", "cth_energy_keep_walls_upload", "cth_restart_write", "cth_restart_wait", "cth_restart_read", "cth_mw_impedance_test", "cth_mw_divergence", "cth_solve_rhoe_pc", "cth_solve_Te_pc", "cth_check_cfl",
    "cth_ion_program_upload", "cth_ion_boxes_upload", "cth_ion_step", "cth_update_neutrals", "cth_fluid_step",
    "cth_batch_steps", "cth_mw_update_create", "cth_mw_update_destroy", "cth_mw_update_due", "cth_mw_update_plane",
    "cth_mw_update_run", "cth_mw_update_prepare", "cth_mw_update_prepared", "cth_update_energy_profile", "cth_mw_port_rescale", "cth_cmat2_mul", "cth_cmat2_inv", "cth_sparam_to_abcd", "cth_abcd_to_sparam", "cth_sparam_setup",
    "cth_unet_create", "cth_unet_destroy", "cth_unet_nparams", "cth_unet_launch_count", "cth_unet_set_tensor_cores", "cth_unet_set_smoothing", "cth_unet_set_wait_test", "cth_unet_set_grid_limit", "cth_unet_check", "cth_unet_set_params", "cth_unet_get_params",
    "cth_unet_get_grads", "cth_unet_set_loss_weights", "cth_unet_forward", "cth_unet_backward",
    "cth_unet_train_step", "cth_unet_set_stats", "cth_unet_features", "cth_unet_predict_dphi",
    "cth_unet_mw_features", "cth_unet_mw_guess", "cth_mw_update_set_net",
)

CTH_PROF_RELAX0 = 0
CTH_PROF_UPDATE = 1
CTH_PROF_RESTRICT0 = 2
CTH_PROF_SETUP = 3
CTH_PROF_RELAXC = 4


class Status(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("nonfinite", ctypes.c_int),
        ("guess", ctypes.c_int),
        ("residual", ctypes.c_double),
        ("initial_residual", ctypes.c_double),
        ("guess_residual", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EnergyParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("dx", "dr", "rmin", "omegam", "masse")]


class EnergyResult(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("Px", "Pr", "Pp", "power_sum")]


class MWPortParams(ctypes.Structure):
    """cth_mw_port_params: the port / reflection / rescale part of update_energy_profile."""
    _fields_ = [(k, ctypes.c_double) for k in ("dx", "dr", "rmin", "omegam", "r1", "r2", "Z0", "Pmw")] + \
        [(k, ctypes.c_double * 2) for k in ("S11", "S21", "S12", "S22")] + \
        [(k, ctypes.c_int) for k in ("flag_mwRef", "i_ref", "j_out", "i_out0", "i_out1", "jf0", "jf1")]


class MWPortResult(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("P_out", "P_fwd", "P_ref", "P_fwd_all", "P_ref_all", "P_err",
                                                 "power_sum", "ratio", "pabs_factor", "field_factor",
                                                 "J1r_exc_factor")] + \
        [(k, ctypes.c_double * 2) for k in ("I_ref", "V_ref", "Gamma_p", "Zp", "Gamma_all", "Zall")]


class CMat2(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double * 2) for k in ("A", "B", "C", "D")]


class SParamParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("S11_mag", "S11_arg_deg", "S21_mag", "S21_arg_deg", "S12_mag",
                                               "S12_arg_deg", "S22_mag", "S22_arg_deg", "Z0", "phase_pre_deg",
                                               "omegam", "epsr_diele", "h0_stab", "dh_stab", "dl_cable")]


class BCList(ctypes.Structure):
    """cth_bc_list: one boundary list of MicrowaveBC (i, j, code arrays)."""
    _fields_ = [("i", ctypes.c_void_p), ("j", ctypes.c_void_p), ("code", ctypes.c_void_p), ("n", ctypes.c_int)]


class MWParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("dx", "dr", "rmin", "omegam", "J1r_exc", "r1", "r2", "masse")]


class TransportParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("masse", "massi", "Ti", "nu_eff", "dTe", "dEi", "dr", "rmin")] + \
               [("flag_Bohm", ctypes.c_int), ("flag_Sagdeev", ctypes.c_int)]


class PhiParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("dt", "dx", "dr", "rmin", "V_bias", "masse", "coefIISEE_ts",
                                               "coefMISEE_ts", "dTe_SEE", "error_cnv_HES_phi",
                                               "error_cnv_SOR_phi")] + \
               [(k, ctypes.c_int) for k in ("maxITR_HES_phi", "maxITR_SOR_phi", "flag_error", "flag_iter_phi",
                                            "precision", "warm_start")] + \
               [("guess_max_relres", ctypes.c_double)]


class PCResult(ctypes.Structure):
    _fields_ = [("ncount", ctypes.c_int), ("solver_rc", ctypes.c_int), ("error_phi", ctypes.c_double),
                ("error_nUex", ctypes.c_double), ("error_nUer", ctypes.c_double),
                ("error_iter", ctypes.c_double * 3), ("solver", Status), ("Ii_Anode", ctypes.c_double),
                ("Ie_Anode", ctypes.c_double), ("I_Anode", ctypes.c_double), ("first", Status)]


class SGParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("dt", "dx", "dr", "rmin", "masse", "coefIISEE_ts", "coefMISEE_ts",
                                               "dTe_SEE", "Te_emitSEE_eV", "ratioEngy_EISEE_rd", "error_cnv_HES",
                                               "error_cnv_SOR")] + \
               [(k, ctypes.c_int) for k in ("maxITR_HES", "maxITR_SOR", "flag_error", "flag_iter", "precision")]


class ImpedanceParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("dx", "dr", "rmin", "omegam", "J1r_exc", "r1", "r2", "Z0", "Pmw")]


class ImpedanceResult(ctypes.Structure):
    _fields_ = [("V", ctypes.c_double * 2), ("I", ctypes.c_double * 2), ("P_fwd", ctypes.c_double),
                ("P_ref", ctypes.c_double), ("ratio", ctypes.c_double), ("J1r_exc_factor", ctypes.c_double),
                ("solve", Status)]


class RestartParams(ctypes.Structure):
    _fields_ = [("dx", ctypes.c_double), ("dr", ctypes.c_double), ("V_bias", ctypes.c_double)]


class RestartInfo(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_int), ("variables_read", ctypes.c_int), ("unknown_columns", ctypes.c_int)]


class CFL(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("CFL", ctypes.c_double), ("masse", ctypes.c_double),
                ("rmin", ctypes.c_double), ("dr", ctypes.c_double), ("flag_adp_dt", ctypes.c_int)] + \
               [(k, ctypes.c_double) for k in ("dt_min", "rhoe_max", "mu_max", "Te_max", "ue_max")]


class IonParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("dt", "dx", "dr", "rmin", "rmax", "massi", "Ti", "V_bias",
                                               "Te_rep_eV", "CFL", "error_cnv_SOR")] + \
               [(k, ctypes.c_int) for k in ("ndt_i", "maxITR_SOR", "flag_iter", "precision", "flag_error")]


class IonResult(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("error_rhoi", "error_Uix", "error_Uir", "error_Uip")] + \
               [("solver_rc", ctypes.c_int), ("reserved", ctypes.c_int), ("solver", Status * 4)]


ION_OP_FIELDS = ("kind", "i0", "i1", "j0", "j1", "di", "dj", "dir", "sign", "bias", "pair", "scale")


class IonOp(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ION_OP_FIELDS]


class NeutralParams(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("dt", "dx", "dr", "rmin", "fn_In", "Tn", "ri", "massi", "DmN",
                                               "error_cnv_SOR")] + \
               [(k, ctypes.c_int) for k in ("ndt_n", "ndt_m", "maxITR_SOR", "flag_iter", "precision", "flag_error",
                                            "n_pos_box")] + [("pos_box", (ctypes.c_int * 4) * 8),
                                                             ("do_rhon", ctypes.c_int), ("do_rhom", ctypes.c_int)]


class NeutralResult(ctypes.Structure):
    _fields_ = [("error_rhon", ctypes.c_double), ("error_rhom", ctypes.c_double), ("solver_rc", ctypes.c_int),
                ("reserved", ctypes.c_int), ("solver", Status * 2)]


class StepParams(ctypes.Structure):
    _fields_ = [("itime", ctypes.c_int), ("ndt_i", ctypes.c_int), ("ndt_n", ctypes.c_int), ("ndt_m", ctypes.c_int),
                ("flag_adp_dt", ctypes.c_int), ("dt", ctypes.c_double), ("CFL", ctypes.c_double),
                ("gtime", ctypes.c_double), ("ion", IonParams), ("phi", PhiParams), ("rhoe", SGParams),
                ("eps", SGParams), ("neutral", NeutralParams), ("transport", TransportParams),
                ("net", ctypes.c_void_p)]


class BatchItem(ctypes.Structure):
    _fields_ = [("fs", ctypes.c_void_p), ("gx", ctypes.c_void_p), ("gr", ctypes.c_void_p),
                ("params", ctypes.POINTER(StepParams)), ("rc", ctypes.c_int), ("steps_done", ctypes.c_int),
                ("seconds", ctypes.c_double), ("I_Anode", ctypes.c_double), ("Ii_Anode", ctypes.c_double),
                ("Ie_Anode", ctypes.c_double), ("mw", ctypes.c_void_p), ("mw_runs", ctypes.c_int),
                ("mw_power_sum", ctypes.c_double), ("mw_J1r_exc", ctypes.c_double)]


class MWUpdateParams(ctypes.Structure):
    """cth_mw_update_params: the microwave update of the time loop."""
    _fields_ = [("mw", MWParams), ("port", MWPortParams), ("ndiv_mw", ctypes.c_int), ("maxit", ctypes.c_int),
                ("tol", ctypes.c_double), ("warm_start", ctypes.c_int)]


class MWUpdateResult(ctypes.Structure):
    _fields_ = [("solve", Status), ("power_sum", ctypes.c_double), ("ratio", ctypes.c_double),
                ("J1r_exc", ctypes.c_double), ("rescale_rc", ctypes.c_int)]


class StepResult(ctypes.Structure):
    _fields_ = [("ion", IonResult), ("phi", PCResult), ("rhoe", PCResult), ("eps", PCResult),
                ("neutral", NeutralResult), ("cfl", CFL), ("ran_ion", ctypes.c_int), ("ran_rhon", ctypes.c_int),
                ("ran_rhom", ctypes.c_int), ("net_ran", ctypes.c_int), ("solver_rc", ctypes.c_int)]


class CathodeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cathode_b200 error {code}: {msg}")
        self.code = code


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_LIB = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the library (raises if it is absent: there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with build.py (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    L.cth_version.restype = ctypes.c_char_p
    L.cth_last_error.restype = ctypes.c_char_p
    L.cth_grid_create.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(_vp)]
    L.cth_grid_create.restype = ctypes.c_int
    L.cth_grid_destroy.argtypes = [_vp]
    L.cth_grid_destroy.restype = None
    L.cth_grid_ld.argtypes = [_vp]
    L.cth_grid_ld.restype = ctypes.c_int
    L.cth_grid_levels.argtypes = [_vp]
    L.cth_grid_levels.restype = ctypes.c_int
    L.cth_c5_solve.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_int, ctypes.c_double, _vp, ctypes.POINTER(Status)]
    L.cth_c5_solve.restype = ctypes.c_int
    L.cth_c5_solve_dev.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_int, ctypes.c_double, _vp, _vp,
                                                       ctypes.POINTER(Status)]
    L.cth_c5_solve_dev.restype = ctypes.c_int
    L.cth_mw_er_assemble_dev.argtypes = [_vp, _vp, _vp, _vp, ctypes.POINTER(MWParams)] + [_vp] * 6 + [_vp]
    L.cth_mw_er_assemble_dev.restype = ctypes.c_int
    L.cth_mw3_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]
    L.cth_mw3_create.restype = ctypes.c_int
    L.cth_mw3_destroy.argtypes = [_vp]
    L.cth_mw3_destroy.restype = None
    L.cth_mw3_ld.argtypes = [_vp]
    L.cth_mw3_ld.restype = ctypes.c_int
    L.cth_mw3_launch_count.argtypes = [_vp]
    L.cth_mw3_launch_count.restype = ctypes.c_longlong
    L.cth_mw3_assemble_dev.argtypes = [_vp] * 6 + [ctypes.POINTER(MWParams), _vp]
    L.cth_mw3_assemble_dev.restype = ctypes.c_int
    L.cth_mw3_copy_planes.argtypes = [_vp, _vp, _vp, _vp]
    L.cth_mw3_copy_planes.restype = ctypes.c_int
    L.cth_mw3_apply_dev.argtypes = [_vp, _vp, _vp, _vp]
    L.cth_mw3_apply_dev.restype = ctypes.c_int
    L.cth_mw3_solve_dev.argtypes = [_vp, ctypes.c_int, ctypes.c_double, _vp, _vp, ctypes.POINTER(Status)]
    L.cth_mw3_solve_dev.restype = ctypes.c_int
    L.cth_mw3_solve_guess_dev.argtypes = [_vp, ctypes.c_int, ctypes.c_double, _vp, _vp, ctypes.c_double, _vp,
                                          ctypes.POINTER(Status)]
    L.cth_mw3_solve_guess_dev.restype = ctypes.c_int
    L.cth_mw3_set_graphs.argtypes = [_vp, ctypes.c_int]
    L.cth_mw3_set_graphs.restype = ctypes.c_int
    L.cth_mw3_create_blocks.argtypes = [ctypes.c_int, ctypes.c_int] + [_vp, _vp, ctypes.c_int] * 3 + \
        [ctypes.c_int, ctypes.POINTER(_vp)]
    L.cth_mw3_create_blocks.restype = ctypes.c_int
    L.cth_mw3_set_boundary.argtypes = [_vp, ctypes.POINTER(BCList), ctypes.c_int]
    L.cth_mw3_set_boundary.restype = ctypes.c_int
    L.cth_mw3_set_precision.argtypes = [_vp, ctypes.c_int]
    L.cth_mw3_set_precision.restype = ctypes.c_int
    L.cth_mw3_assemble_explicit_dev.argtypes = [_vp, _vp, _vp, _vp, _vp, ctypes.POINTER(MWParams), _vp]
    L.cth_mw3_assemble_explicit_dev.restype = ctypes.c_int
    L.cth_mw3_fill_ghosts.argtypes = [_vp, _vp, _vp, _vp, ctypes.POINTER(MWParams), _vp]
    L.cth_mw3_fill_ghosts.restype = ctypes.c_int
    L.cth_mw3_set_cycle.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.cth_mw3_set_cycle.restype = ctypes.c_int
    L.cth_mw3_set_preconditioner.argtypes = [_vp, ctypes.c_int]
    L.cth_mw3_set_preconditioner.restype = ctypes.c_int
    L.cth_fields_create.argtypes = [_vp, ctypes.POINTER(_vp)]
    L.cth_fields_create.restype = ctypes.c_int
    L.cth_fields_destroy.argtypes = [_vp]
    L.cth_fields_destroy.restype = None
    L.cth_field.argtypes = [_vp, ctypes.c_char_p]
    L.cth_field.restype = ctypes.c_void_p
    L.cth_field_upload.argtypes = [_vp, ctypes.c_char_p, _vp]
    L.cth_field_upload.restype = ctypes.c_int
    L.cth_field_download.argtypes = [_vp, ctypes.c_char_p, _vp]
    L.cth_field_download.restype = ctypes.c_int
    L.cth_flags_upload.argtypes = [_vp, _vp]
    L.cth_flags_upload.restype = ctypes.c_int
    L.cth_table_upload.argtypes = [_vp, ctypes.c_char_p, _vp, ctypes.c_int]
    L.cth_table_upload.restype = ctypes.c_int
    L.cth_update_transport_coef.argtypes = [_vp, ctypes.POINTER(TransportParams), _vp]
    L.cth_update_transport_coef.restype = ctypes.c_int
    L.cth_solve_phi_pc.argtypes = [_vp, ctypes.POINTER(PhiParams), _vp, ctypes.POINTER(PCResult)]
    L.cth_solve_phi_pc.restype = ctypes.c_int
    L.cth_ion_program_upload.argtypes = [_vp, ctypes.c_int, _vp, ctypes.c_int]
    L.cth_ion_program_upload.restype = ctypes.c_int
    L.cth_ion_boxes_upload.argtypes = [_vp, ctypes.c_int, _vp, ctypes.c_int]
    L.cth_ion_boxes_upload.restype = ctypes.c_int
    L.cth_ion_step.argtypes = [_vp, _vp, _vp, ctypes.POINTER(IonParams), _vp, ctypes.POINTER(IonResult)]
    L.cth_ion_step.restype = ctypes.c_int
    L.cth_update_neutrals.argtypes = [_vp, ctypes.POINTER(NeutralParams), _vp, ctypes.POINTER(NeutralResult)]
    L.cth_update_neutrals.restype = ctypes.c_int
    L.cth_fluid_step.argtypes = [_vp, _vp, _vp, ctypes.POINTER(StepParams), _vp, ctypes.POINTER(StepResult)]
    L.cth_fluid_step.restype = ctypes.c_int
    L.cth_check_cfl.argtypes = [_vp, ctypes.POINTER(CFL), _vp]
    L.cth_check_cfl.restype = ctypes.c_int
    L.cth_ghost_rules_upload.argtypes = [_vp, _vp, ctypes.c_int]
    L.cth_ghost_rules_upload.restype = ctypes.c_int
    L.cth_energy_keep_walls_upload.argtypes = [_vp, _vp, ctypes.c_int]
    L.cth_energy_keep_walls_upload.restype = ctypes.c_int
    L.cth_mw_impedance_test.argtypes = [_vp, _vp, ctypes.POINTER(ImpedanceParams), ctypes.c_int, ctypes.c_double,
                                        _vp, _vp, ctypes.POINTER(ImpedanceResult)]
    L.cth_mw_impedance_test.restype = ctypes.c_int
    L.cth_mw_divergence.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_double] * 4 + [_vp] * 3 + \
        [ctypes.POINTER(ctypes.c_double), _vp]
    L.cth_mw_divergence.restype = ctypes.c_int
    L.cth_restart_write.argtypes = [_vp, ctypes.c_char_p, _vp, _vp, _vp]
    L.cth_restart_write.restype = ctypes.c_int
    L.cth_restart_wait.argtypes = [_vp]
    L.cth_restart_wait.restype = ctypes.c_int
    L.cth_restart_read.argtypes = [_vp, _vp, _vp, ctypes.c_char_p, _vp, _vp, ctypes.POINTER(RestartParams), _vp,
                                   ctypes.POINTER(RestartInfo)]
    L.cth_restart_read.restype = ctypes.c_int
    for nm in ("cth_solve_rhoe_pc", "cth_solve_Te_pc"):
        getattr(L, nm).argtypes = [_vp, ctypes.POINTER(SGParams), _vp, ctypes.POINTER(PCResult)]
        getattr(L, nm).restype = ctypes.c_int
    L.cth_grid_set_graphs.argtypes = [_vp, ctypes.c_int]
    L.cth_grid_set_graphs.restype = ctypes.c_int
    L.cth_grid_time_relax.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.cth_grid_time_relax.restype = ctypes.c_int
    L.cth_grid_set_tail.argtypes = [_vp, ctypes.c_int]
    L.cth_grid_set_tail.restype = ctypes.c_int
    L.cth_grid_time_cycle.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.cth_grid_time_cycle.restype = ctypes.c_int
    L.cth_grid_set_reuse.argtypes = [_vp, ctypes.c_double, ctypes.c_int]
    L.cth_grid_set_reuse.restype = ctypes.c_int
    L.cth_grid_reuse_stats.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.cth_grid_reuse_stats.restype = ctypes.c_int
    L.cth_grid_set_cycle.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.cth_grid_set_cycle.restype = ctypes.c_int
    L.cth_smg_solve.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp,
                                                    ctypes.POINTER(Status)]
    L.cth_smg_solve.restype = ctypes.c_int
    L.cth_smg_solve_dev.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                        _vp, _vp, ctypes.POINTER(Status)]
    L.cth_smg_solve_dev.restype = ctypes.c_int
    L.cth_smg_solve_guess_dev.argtypes = [_vp] + [_vp] * 7 + [ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                                              ctypes.c_int, _vp, _vp, ctypes.POINTER(Status)]
    L.cth_smg_solve_guess_dev.restype = ctypes.c_int
    for f in ("cth_fields_upload_many", "cth_fields_download_many"):
        getattr(L, f).argtypes = [_vp, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(_vp), ctypes.c_int, _vp]
        getattr(L, f).restype = ctypes.c_int
    L.cth_fields_set_warm_start.argtypes = [_vp, ctypes.c_int, ctypes.c_double]
    L.cth_fields_set_warm_start.restype = ctypes.c_int
    L.cth_fields_set_download_plan.argtypes = [_vp, _vp, _vp, ctypes.c_int]
    L.cth_fields_set_download_plan.restype = ctypes.c_int
    L.cth_fields_download_wait.argtypes = [_vp]
    L.cth_fields_download_wait.restype = ctypes.c_int
    L.cth_fields_set_upload_plan.argtypes = [_vp, _vp, _vp, ctypes.c_int]
    L.cth_fields_set_upload_plan.restype = ctypes.c_int
    L.cth_batch_steps.argtypes = [ctypes.POINTER(BatchItem), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double)]
    L.cth_batch_steps.restype = ctypes.c_int
    L.cth_mw_update_create.argtypes = [_vp, _vp, ctypes.POINTER(MWUpdateParams), _vp, _vp, ctypes.POINTER(_vp)]
    L.cth_mw_update_create.restype = ctypes.c_int
    L.cth_mw_update_destroy.argtypes = [_vp]
    L.cth_mw_update_destroy.restype = None
    L.cth_mw_update_due.argtypes = [_vp, ctypes.c_int]
    L.cth_mw_update_due.restype = ctypes.c_int
    L.cth_mw_update_plane.argtypes = [_vp, ctypes.c_int]
    L.cth_mw_update_plane.restype = ctypes.c_void_p
    L.cth_mw_update_run.argtypes = [_vp, _vp, _vp, _vp, ctypes.POINTER(MWUpdateResult)]
    L.cth_mw_update_run.restype = ctypes.c_int
    L.cth_mw_update_prepare.argtypes = [_vp, _vp]
    L.cth_mw_update_prepare.restype = ctypes.c_int
    L.cth_mw_update_prepared.argtypes = [_vp]
    L.cth_mw_update_prepared.restype = ctypes.c_int
    L.cth_update_energy_profile.argtypes = [_vp, _vp, _vp, ctypes.POINTER(EnergyParams)] + [_vp] * 7 + \
        [ctypes.POINTER(EnergyResult)]
    L.cth_update_energy_profile.restype = ctypes.c_int
    L.cth_mw_port_rescale.argtypes = [_vp, ctypes.POINTER(MWPortParams), ctypes.c_double] + [_vp] * 10 + \
        [ctypes.POINTER(MWPortResult)]
    L.cth_mw_port_rescale.restype = ctypes.c_int
    _c2 = ctypes.c_double * 2
    L.cth_cmat2_mul.argtypes = [ctypes.POINTER(CMat2)] * 3
    L.cth_cmat2_mul.restype = ctypes.c_int
    L.cth_cmat2_inv.argtypes = [ctypes.POINTER(CMat2)] * 2
    L.cth_cmat2_inv.restype = ctypes.c_int
    L.cth_sparam_to_abcd.argtypes = [ctypes.POINTER(_c2)] * 4 + [ctypes.c_double, ctypes.POINTER(CMat2)]
    L.cth_sparam_to_abcd.restype = ctypes.c_int
    L.cth_abcd_to_sparam.argtypes = [ctypes.POINTER(CMat2), ctypes.c_double] + [ctypes.POINTER(_c2)] * 4
    L.cth_abcd_to_sparam.restype = ctypes.c_int
    L.cth_sparam_setup.argtypes = [ctypes.POINTER(SParamParams), ctypes.POINTER(_c2 * 4),
                                   ctypes.POINTER(ctypes.c_double)]
    L.cth_sparam_setup.restype = ctypes.c_int
    L.cth_unet_create.argtypes = [ctypes.c_int] * 6
    L.cth_unet_create.restype = _vp
    L.cth_unet_destroy.argtypes = [_vp]
    L.cth_unet_destroy.restype = None
    L.cth_unet_nparams.argtypes = [_vp]
    L.cth_unet_nparams.restype = ctypes.c_longlong
    L.cth_unet_set_tensor_cores.argtypes = [_vp, ctypes.c_int]
    L.cth_unet_set_tensor_cores.restype = ctypes.c_int
    L.cth_unet_set_smoothing.argtypes = [_vp, ctypes.c_int]
    L.cth_unet_set_smoothing.restype = ctypes.c_int
    L.cth_unet_set_wait_test.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.cth_unet_set_wait_test.restype = ctypes.c_int
    L.cth_unet_set_grid_limit.argtypes = [_vp, ctypes.c_int]
    L.cth_unet_set_grid_limit.restype = ctypes.c_int
    L.cth_unet_check.argtypes = [_vp]
    L.cth_unet_check.restype = ctypes.c_int
    L.cth_unet_launch_count.argtypes = [_vp]
    L.cth_unet_launch_count.restype = ctypes.c_longlong
    for f in ("cth_unet_set_params", "cth_unet_get_params", "cth_unet_get_grads"):
        getattr(L, f).argtypes = [_vp, _vp, ctypes.c_longlong]
        getattr(L, f).restype = ctypes.c_int
    for f in ("cth_unet_set_loss_weights", "cth_unet_set_stats"):
        getattr(L, f).argtypes = [_vp, _vp]
        getattr(L, f).restype = ctypes.c_int
    L.cth_unet_forward.argtypes = [_vp, _vp, _vp, _vp]
    L.cth_unet_forward.restype = ctypes.c_int
    L.cth_unet_backward.argtypes = [_vp, _vp, _vp]
    L.cth_unet_backward.restype = ctypes.c_int
    L.cth_unet_train_step.argtypes = [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_float, ctypes.c_int, _vp,
                                      ctypes.POINTER(ctypes.c_double)]
    L.cth_unet_train_step.restype = ctypes.c_int
    L.cth_unet_features.argtypes = [_vp, _vp, _vp, _vp]
    L.cth_unet_features.restype = ctypes.c_int
    L.cth_unet_predict_dphi.argtypes = [_vp, _vp, _vp]
    L.cth_unet_predict_dphi.restype = ctypes.c_int
    L.cth_unet_mw_features.argtypes = [_vp, _vp, _vp, ctypes.c_double, _vp, _vp]
    L.cth_unet_mw_features.restype = ctypes.c_int
    L.cth_unet_mw_guess.argtypes = [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp, _vp]
    L.cth_unet_mw_guess.restype = ctypes.c_int
    L.cth_mw_update_set_net.argtypes = [_vp, _vp]
    L.cth_mw_update_set_net.restype = ctypes.c_int
    L.cth_sor_solve.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_double, ctypes.c_int, ctypes.c_double, _vp,
                                                    ctypes.POINTER(Status)]
    L.cth_sor_solve.restype = ctypes.c_int
    L.cth_sor_solve_dev.argtypes = [_vp] + [_vp] * 6 + [ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                                        _vp, _vp, ctypes.POINTER(Status)]
    L.cth_sor_solve_dev.restype = ctypes.c_int
    L.cth_residual_dev.argtypes = [_vp] + [_vp] * 7 + [_vp, _dp, _dp, _vp]
    L.cth_residual_dev.restype = ctypes.c_int
    L.cth_to_device_layout.argtypes = [_vp, _vp, _vp, _vp]
    L.cth_to_device_layout.restype = ctypes.c_int
    L.cth_from_device_layout.argtypes = [_vp, _vp, _vp, _vp]
    L.cth_from_device_layout.restype = ctypes.c_int
    L.cth_residual_noalloc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int] + \
        [_vp] * 8 + [_dp, _dp, _vp]
    L.cth_residual_noalloc.restype = ctypes.c_int
    L.cth_launch_count.argtypes = [_vp]
    L.cth_launch_count.restype = ctypes.c_longlong
    L.cth_profile.argtypes = [_vp, ctypes.c_int]
    L.cth_profile.restype = ctypes.c_int
    L.cth_profile_read.argtypes = [_vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_longlong), _dp]
    L.cth_profile_read.restype = ctypes.c_int
    _LIB = L
    return L


def last_error() -> str:
    return load().cth_last_error().decode()


def check(rc: int, allow_positive: bool = True) -> int:
    if rc < 0 or (rc > 0 and not allow_positive):
        raise CathodeError(rc, last_error())
    return rc
