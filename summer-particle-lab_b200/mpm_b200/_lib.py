"""ctypes binding of libmpm_b200.so (the C ABI declared in include/mpm_b200.h).

The library is built in-tree by summer-particle-lab_b200/build_lib.py. There is no CPU fallback:
if the shared object is missing or cannot be loaded, every entry point raises.
"""
import ctypes
import os

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libmpm_b200.so")

_D = ctypes.c_double
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_P = ctypes.c_void_p

OK = 0
ERRORS = {
    -1: "MPM_ERR_INVALID_ARG", -2: "MPM_ERR_OUT_OF_MEMORY", -3: "MPM_ERR_CUDA", -4: "MPM_ERR_NONFINITE",
    -5: "MPM_ERR_INVALID_J", -6: "MPM_ERR_OUT_OF_RANGE", -7: "MPM_ERR_TIMEOUT", -8: "MPM_ERR_STATE",
    -9: "MPM_ERR_CAPACITY", -10: "MPM_ERR_UNSUPPORTED",
}
STATUS_NONFINITE, STATUS_INVALID_J, STATUS_OUT_OF_RANGE, STATUS_TIMEOUT, STATUS_SCATTER_OVERFLOW = 1, 2, 4, 8, 16
F64, F32 = 0, 1
PROFILE_KERNELS = ("begin", "grid_update", "g2p2g", "scan", "sort_scatter", "p2g", "keys")


class MpmDomain(ctypes.Structure):
    _fields_ = [("lower", _D * 3), ("upper", _D * 3), ("cell_size", _D), ("gravity", _D * 3),
                ("sticky_floor", _I32), ("clamp_positions", _I32), ("mass_eps", _D), ("cfl", _D),
                ("dt_max", _D), ("grad_limit", _D), ("cubic", _I32), ("reserved", _I32)]


class MpmMaterial(ctypes.Structure):
    _fields_ = [("model", _I32), ("reserved", _I32), ("mu", _D), ("lam", _D), ("yield_stress", _D),
                ("hardening", _D), ("T_ref", _D), ("T_hot", _D), ("hot_ratio", _D),
                ("heat_fraction", _D), ("specific_heat", _D),
                ("jc_n", _D), ("jc_C", _D), ("jc_rate0", _D), ("T_melt", _D), ("jc_m", _D),
                ("creep_rate", _D), ("creep_Q", _D), ("creep_n", _D), ("creep_stress", _D),
                ("temperature_offset", _D), ("yield_strain", _D), ("friction_deg", _D),
                ("dp_cohesion", _D), ("dp_slope", _D), ("dp_dilatancy", _D), ("dp_tension", _D),
                ("df_alpha", _D), ("df_plateau", _D), ("df_gamma", _D), ("df_densify", _D), ("df_beta", _D),
                ("df_eps_d", _D), ("conductivity", _D), ("melting_point", _D), ("latent_heat", _D)]


class MpmRegularizer(ctypes.Structure):
    _fields_ = [("enabled", _I32), ("reserved", _I32), ("spacing", _D), ("volume_unit", _D), ("max_speed", _D),
                ("rate", _D)]


class MpmParticles(ctypes.Structure):
    _fields_ = [("dtype", _I32), ("reserved", _I32), ("x", _P), ("y", _P), ("z", _P), ("vx", _P),
                ("vy", _P), ("vz", _P), ("mass", _P), ("volume", _P), ("temperature", _P),
                ("plastic", _P), ("F", _P), ("C", _P), ("material", _P), ("pinned", _P), ("jp", _P),
                ("dilation", _P), ("enthalpy", _P), ("melted", _P)]


class MpmHeatExchange(ctypes.Structure):
    _fields_ = [("radius", _D), ("geometry", _D), ("heat_rate", _D), ("ambient", _I32), ("reserved", _I32),
                ("ambient_T", _D), ("ambient_rate", _D)]


class MpmLedger(ctypes.Structure):
    _fields_ = [("mass", _D), ("kinetic", _D), ("affine", _D), ("potential", _D), ("elastic", _D),
                ("momentum", _D * 3), ("angular", _D * 3), ("min_j", _D), ("max_j", _D),
                ("max_plastic", _D), ("max_von_mises", _D), ("plastic_work", _D), ("count", _I64),
                ("nonfinite", _I64), ("invalid_j", _I64)]


class MpmSceneDesc(ctypes.Structure):
    _fields_ = [("domain", MpmDomain), ("material", _I32), ("reserved", _I32), ("count", _I64)]


class MpmTuning(ctypes.Structure):
    _fields_ = [("warp_specialised", _I32), ("reserved", _I32), ("blocks_per_sm", _I32),
                ("reorder_interval", _I32), ("use_tma", _I32), ("trials", _I32),
                ("ms_per_substep", _D), ("ms_per_substep_default", _D)]


class MpmSurrogateConfig(ctypes.Structure):
    _fields_ = [("samples", _I64), ("batch", _I32), ("steps", _I32), ("lr", _D), ("weight_decay", _D),
                ("dep_weight", _D), ("cosine", _I32), ("newton", _I32), ("seed", ctypes.c_uint64),
                ("strain_min", _D), ("strain_max", _D), ("T_min", _D), ("T_max", _D), ("ep_max", _D),
                ("dt_min", _D), ("dt_max", _D)]


class MpmGateCounts(ctypes.Structure):
    _fields_ = [("elastic", ctypes.c_uint32), ("learned", ctypes.c_uint32), ("fallback", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


SURROGATE_PARAMS = 5768
RETURN_EXACT, RETURN_LEARNED_GATED, RETURN_NEWTON_GATED = 0, 1, 2


class MpmFrameInfo(ctypes.Structure):
    _fields_ = [("count", _I64), ("rows", _I64), ("stride", _I64), ("mass", _D), ("thermal_energy", _D),
                ("min_T", _D), ("max_T", _D), ("min_j", _D), ("max_von_mises", _D), ("max_plastic", _D),
                ("nonfinite", _I64), ("per_material", _I64 * 256)]


class SmpmSim(ctypes.Structure):
    _fields_ = [("count", _I32), ("scene", _I32), ("boundary", _I32), ("gravity", _I32),
                ("solid_stiffness", _D), ("strength", _D), ("x", _P), ("y", _P), ("vx", _P), ("vy", _P),
                ("mass", _P), ("volume", _P), ("material", _P), ("pinned", _P)]


class SmpmStats(ctypes.Structure):
    _fields_ = [("count", _I32), ("nodes", _I32), ("substeps", _I32), ("pad", _I32), ("min_j", _D),
                ("max_j", _D), ("strain", _D)]


SMPM_SCENES = {"softbody": 1, "basin": 2}
SMPM_GRAVITY = {"none": 0, "center": 1, "uniform": 2}

# name -> (restype, argtypes)
SIGNATURES = {
    "mpm_abi_version": (ctypes.c_int, []),
    "mpm_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "mpm_create": (ctypes.c_int, [ctypes.POINTER(MpmDomain), _I64, ctypes.POINTER(_P)]),
    "mpm_destroy": (ctypes.c_int, [_P]),
    "mpm_last_error": (ctypes.c_char_p, [_P]),
    "mpm_configure_domain": (ctypes.c_int, [_P, ctypes.POINTER(MpmDomain)]),
    "mpm_grid_dims": (ctypes.c_int, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_D)]),
    "mpm_set_material": (ctypes.c_int, [_P, _I32, ctypes.POINTER(MpmMaterial)]),
    "mpm_validate_material": (ctypes.c_int, [ctypes.POINTER(MpmMaterial)]),
    "mpm_set_regularizer": (ctypes.c_int, [_P, ctypes.POINTER(MpmRegularizer)]),
    "mpm_regularize": (ctypes.c_int, [_P, _D]),
    "mpm_regularize_host": (ctypes.c_int, [_P, ctypes.POINTER(MpmParticles), _D]),
    "mpm_exchange_heat": (ctypes.c_int, [_P, ctypes.POINTER(MpmHeatExchange), _D, ctypes.POINTER(_D)]),
    "mpm_batch_set_slabs": (ctypes.c_int, [_P, _I32]),
    "mpm_set_open_faces": (ctypes.c_int, [_P, _I32]),
    "mpm_prepare": (ctypes.c_int, [_P]),
    "mpm_halo_bytes": (ctypes.c_int, [_P, _I32, ctypes.POINTER(_I64)]),
    "mpm_halo_export": (ctypes.c_int, [_P, _I32, _I32, _P]),
    "mpm_halo_add": (ctypes.c_int, [_P, _I32, _I32, _P]),
    "mpm_get_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "mpm_upload_particles": (ctypes.c_int, [_P, _I64, ctypes.POINTER(MpmParticles)]),
    "mpm_download_particles": (ctypes.c_int, [_P, ctypes.POINTER(MpmParticles)]),
    "mpm_count": (ctypes.c_int, [_P, ctypes.POINTER(_I64)]),
    "mpm_reset_deformation": (ctypes.c_int, [_P]),
    "mpm_stable_dt": (ctypes.c_int, [_P, ctypes.POINTER(_D)]),
    "mpm_step": (ctypes.c_int, [_P, _D, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_D)]),
    "mpm_step_fixed": (ctypes.c_int, [_P, _D, _I32]),
    "mpm_step_cfl": (ctypes.c_int, [_P, _I32, ctypes.POINTER(_D)]),
    "mpm_step_host": (ctypes.c_int, [_P, ctypes.POINTER(MpmParticles), _D]),
    "mpm_frame_host": (ctypes.c_int, [_P, ctypes.POINTER(MpmParticles), _D, _I32, ctypes.POINTER(_I32)]),
    "mpm_check_bounded_wait": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.POINTER(_I32)]),
    "mpm_run": (ctypes.c_int, [_P, _D, _I32, _I32, ctypes.POINTER(_I32), ctypes.POINTER(_D)]),
    "mpm_profile_enable": (ctypes.c_int, [_P, _I32]),
    "mpm_profile_read": (ctypes.c_int, [_P, ctypes.POINTER(_D), ctypes.POINTER(_I64)]),
    "mpm_launch_count": (ctypes.c_int, [_P, ctypes.POINTER(_I64)]),
    "mpm_ledger_compute": (ctypes.c_int, [_P, ctypes.POINTER(MpmLedger)]),
    "mpm_min_j": (ctypes.c_int, [_P, ctypes.POINTER(_D)]),
    "mpm_status": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint32)]),
    "mpm_clear_status": (ctypes.c_int, [_P]),
    "mpm_grid_debug": (ctypes.c_int, [_P, _D, _P, _P]),
    "mpm_snapshot": (ctypes.c_int, [_P]),
    "mpm_rollback": (ctypes.c_int, [_P]),
    "mpm_checkpoint_save": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "mpm_checkpoint_load": (ctypes.c_int, [_P, ctypes.c_char_p]),
    "mpm_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(_P)]),
    "mpm_host_free": (ctypes.c_int, [_P]),
    "mpm_return_map_batch": (ctypes.c_int, [ctypes.POINTER(MpmMaterial), _I64, _P, _P, _P, _D, _P, _P, _P]),
    "mpm_p2g_noalloc": (ctypes.c_int, [ctypes.POINTER(MpmDomain), ctypes.POINTER(MpmMaterial), _I64, _P, _P, _P, _P, _P,
                                        _P, _D, _P, _P, _P]),
    "mpm_pack_frame": (ctypes.c_int, [_P, _I64, _P, _I64, ctypes.POINTER(MpmFrameInfo)]),
    "mpm_set_conduction": (ctypes.c_int, [_P, _I32, _D, _D, _D]),
    "mpm_reset_particle": (ctypes.c_int, [_P, _I64]),
    "mpm_remove_particle": (ctypes.c_int, [_P, _I64, _I64]),
    "mpm_batch_create": (ctypes.c_int, [ctypes.POINTER(MpmSceneDesc), _I32, ctypes.POINTER(_P)]),
    "mpm_batch_count": (ctypes.c_int, [_P, ctypes.POINTER(_I32)]),
    "mpm_batch_run": (ctypes.c_int, [_P, _I32, _I32]),
    "mpm_batch_times": (ctypes.c_int, [_P, _P, _P]),
    "mpm_batch_ledger": (ctypes.c_int, [_P, _I32, ctypes.POINTER(MpmLedger)]),
    "mpm_batch_grid_debug": (ctypes.c_int, [_P, _I32, _D, _P, _P]),
    "mpm_batch_autotune": (ctypes.c_int, [_P, _I32, ctypes.POINTER(MpmTuning)]),
    "mpm_surrogate_create": (ctypes.c_int, [ctypes.POINTER(MpmMaterial), ctypes.c_uint64, ctypes.POINTER(_P)]),
    "mpm_surrogate_destroy": (ctypes.c_int, [_P]),
    "mpm_surrogate_last_error": (ctypes.c_char_p, [_P]),
    "mpm_surrogate_get_weights": (ctypes.c_int, [_P, _P]),
    "mpm_surrogate_set_weights": (ctypes.c_int, [_P, _P]),
    "mpm_surrogate_samples": (ctypes.c_int, [_P, ctypes.POINTER(MpmSurrogateConfig), _I64, _P, _P, _P, _P, _P]),
    "mpm_surrogate_train": (ctypes.c_int, [_P, ctypes.POINTER(MpmSurrogateConfig), _P]),
    "mpm_surrogate_grad": (ctypes.c_int, [_P, _I64, _P, _P, _P, _P, ctypes.POINTER(_D)]),
    "mpm_surrogate_forward": (ctypes.c_int, [_P, _I64, _P, _P]),
    "mpm_return_map_learned": (ctypes.c_int, [_P, _I64, _P, _P, _P, _D, _I32, _P, _P, _P, _P,
                                               ctypes.POINTER(MpmGateCounts)]),
    "mpm_surrogate_time": (ctypes.c_int, [_P, ctypes.POINTER(MpmSurrogateConfig), _I64, _I32, _D, ctypes.POINTER(_D),
                                           ctypes.POINTER(_D), ctypes.POINTER(MpmGateCounts)]),
    "mpm_surrogate_time_newton": (ctypes.c_int, [_P, ctypes.POINTER(MpmSurrogateConfig), _I64, _I32, _D,
                                                  ctypes.POINTER(_D), ctypes.POINTER(MpmGateCounts)]),
    "mpm_set_return_mode": (ctypes.c_int, [_P, _I32, _P, _D, _I32]),
    "mpm_gate_counts_read": (ctypes.c_int, [_P, ctypes.POINTER(MpmGateCounts), _I32]),
    "smpm_create": (ctypes.c_int, [_I64, ctypes.POINTER(_P)]),
    "smpm_destroy": (ctypes.c_int, [_P]),
    "smpm_last_error": (ctypes.c_char_p, [_P]),
    "smpm_set_mpm_materials": (ctypes.c_int, [_P, _P, _I32]),
    "smpm_reset": (ctypes.c_int, [_P]),
    "smpm_reset_particle": (ctypes.c_int, [_P, _I64]),
    "smpm_remove_particle": (ctypes.c_int, [_P, _I64, _I64]),
    "smpm_has_particles": (ctypes.c_int, [_P, ctypes.POINTER(SmpmSim), ctypes.POINTER(_I32)]),
    "smpm_stable_step": (ctypes.c_int, [_P, ctypes.POINTER(SmpmSim), ctypes.POINTER(_D)]),
    "smpm_step": (ctypes.c_int, [_P, ctypes.POINTER(SmpmSim), _D]),
    "smpm_stats_get": (ctypes.c_int, [_P, ctypes.POINTER(SmpmSim), ctypes.POINTER(SmpmStats)]),
    "smpm_frame": (ctypes.c_int, [_P, ctypes.POINTER(SmpmSim), _D, ctypes.POINTER(_I32), ctypes.POINTER(_D)]),
    "smpm_get_fields": (ctypes.c_int, [_P, _I64, _P]),
    "smpm_set_fields": (ctypes.c_int, [_P, _I64, _P]),
}

_lib = None


class MpmError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


def lib():
    """The loaded library. Raises when the in-tree build is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python __graft_entry__.py build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc, handle=None):
    if rc != OK:
        msg = lib().mpm_last_error(handle).decode() if handle else lib().mpm_error_string(rc).decode()
        raise MpmError(rc, msg)
    return rc


def check2(rc, handle=None):
    """check() for the 2D (smpm_*) handles."""
    if rc != OK:
        msg = lib().smpm_last_error(handle).decode() if handle else lib().mpm_error_string(rc).decode()
        raise MpmError(rc, msg)
    return rc
