"""ctypes binding of libmonoalg3d_b200.so (include/monoalg3d_b200.h).

The shared library is built in-tree by ``monoalg3d_c_b200/csrc/Makefile`` and
loaded at the first call into it.  There is no fallback: if the library is
missing, that call raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmonoalg3d_b200.so")

MB_OK = 0
MB_ERR_ARG = 1
MB_ERR_CUDA = 2
MB_ERR_NAN = 3
MB_ERR_NOMEM = 4
MB_ERR_UNSUPPORTED = 5
MB_ERR_STATE = 6

MB_MODEL_TT2006 = 0
MB_MODEL_TORORD_FKATP_MIXED = 1
MB_MODEL_TORORD_FKATP_ENDO = 2
MB_ODE_FIXED = 0
MB_ODE_ADAPTIVE_CPU = 1
MB_ODE_ADAPTIVE_GPU = 2
MB_PREC_FP64 = 0
MB_PREC_MIXED = 1
MB_RL_REFERENCE_CPU = 0
MB_RL_TRUE = 1
MB_STIM_X_LESS_THAN = 0
MB_STIM_X_Y_LIMITS = 1
MB_STIM_X_Y_Z_LIMITS = 2
MB_STIM_CELL_MASK = 3
MB_ASSEMBLY_HOMOGENEOUS = 0
MB_ASSEMBLY_ANISOTROPIC = 1
MB_ASSEMBLY_PER_CELL_SIGMA = 2
MB_MAX_STIMS = 8
MB_NUM_SCALES = 5

# Every symbol include/monoalg3d_b200.h declares.
EXPORTED = [
    "mb_last_error", "mb_version", "mb_device_count", "mb_init_cell_model_data",
    "mb_ode_create", "mb_set_model_initial_conditions_gpu", "mb_solve_model_odes_gpu",
    "mb_ode_get_state", "mb_ode_set_state", "mb_ode_set_v", "mb_ode_get_v", "mb_ode_destroy",
    "mb_csr_create", "mb_csr_solve", "mb_csr_destroy",
    "mb_monodomain_desc_defaults", "mb_monodomain_create", "mb_monodomain_destroy",
    "mb_monodomain_step", "mb_monodomain_sync", "mb_solve_all_volumes_odes",
    "mb_update_monodomain_default", "mb_conjugate_gradient", "mb_advance_time",
    "mb_monodomain_step_host", "mb_monodomain_get_v", "mb_monodomain_set_v", "mb_monodomain_get_activation",
    "mb_monodomain_get_ecg", "mb_monodomain_step_host_async", "mb_monodomain_host_wait",
    "mb_monodomain_time_steps_host_async",
    "mb_batch_pack", "mb_monodomain_checkpoint_bytes", "mb_monodomain_checkpoint", "mb_monodomain_restore",
    "mb_monodomain_save_v", "mb_adjoint_create", "mb_adjoint_forward", "mb_adjoint_backward", "mb_adjoint_destroy",
    "mb_monodomain_get_state", "mb_monodomain_info", "mb_monodomain_step_stats",
    "mb_monodomain_device_v", "mb_monodomain_profile_steps", "mb_csr_conjugate_gradient",
    "mb_monodomain_tuning", "mb_monodomain_time_steps", "mb_monodomain_time_steps_host",
    "mb_csr_conjugate_gradient_noalloc", "mb_cg_launch_shapes",
    "mb_monodomain_save_state", "mb_monodomain_restore_state", "mb_reference_cell_order",
    "mb_torord_endo_initial_state", "mb_torord_initial_state", "mb_ode_device_state", "mb_ode_set_steps",
]


class MbStim(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("start", C.c_double),
        ("duration", C.c_double),
        ("period", C.c_double),
        ("current", C.c_double),
        ("x_limit", C.c_double),
        ("min", C.c_double * 3),
        ("max", C.c_double * 3),
        ("cell_mask", C.c_void_p),
    ]


class MbDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("active", C.c_void_p),
        ("dt_pde", C.c_double), ("beta", C.c_double), ("cm", C.c_double),
        ("model", C.c_int), ("precision", C.c_int), ("rl_rule", C.c_int),
        ("dt_ode", C.c_double),
        ("initial_state", C.c_void_p),
        ("celltype", C.c_void_p),
        ("current_scale", C.c_void_p),
        ("assembly", C.c_int),
        ("sigma", C.c_double * 3),
        ("sigma_l", C.c_double), ("sigma_t", C.c_double), ("sigma_n", C.c_double),
        ("fibre_angle_z", C.c_void_p),
        ("sigma_cell", C.c_void_p),
        ("cg_tolerance", C.c_double),
        ("cg_max_iterations", C.c_int),
        ("use_preconditioner", C.c_int),
        ("num_stims", C.c_int),
        ("stims", MbStim * MB_MAX_STIMS),
        ("initial_v", C.c_double),
        ("track_activation", C.c_int),
        ("activation_threshold", C.c_double),
        ("activation_min_interval", C.c_double),
        ("ecg_rate", C.c_int),
        ("ecg_n_leads", C.c_int),
        ("ecg_leads", C.c_void_p),
        ("ecg_sigma_b", C.c_double),
        ("ecg_capacity", C.c_int64),
        ("ode_adaptive", C.c_int),
        ("ode_abs_tol", C.c_double),
        ("ode_rel_tol", C.c_double),
    ]


class MbStepStats(C.Structure):
    _fields_ = [("cg_iterations", C.c_int32), ("refinements", C.c_int32), ("cg_error", C.c_double)]


class MonoAlgError(RuntimeError):
    """A non-zero status from the C ABI; .code holds the MB_ERR_* value."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C monoalg3d_c_b200/csrc` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    vp, i32, u32, i64, dbl = C.c_void_p, C.c_int, C.c_uint32, C.c_int64, C.c_double
    P = C.POINTER
    sig = {
        "mb_last_error": (C.c_char_p, []),
        "mb_version": (i32, []),
        "mb_device_count": (i32, [P(i32)]),
        "mb_init_cell_model_data": (i32, [i32, P(i32), P(dbl)]),
        "mb_ode_create": (i32, [P(vp), i32, i32, i32, u32, dbl, u32]),
        "mb_set_model_initial_conditions_gpu": (i32, [vp, vp, vp, P(C.c_size_t)]),
        "mb_solve_model_odes_gpu": (i32, [vp, dbl, vp]),
        "mb_ode_get_state": (i32, [vp, vp]),
        "mb_ode_set_state": (i32, [vp, vp]),
        "mb_ode_set_v": (i32, [vp, vp, C.c_size_t]),
        "mb_ode_get_v": (i32, [vp, vp, C.c_size_t]),
        "mb_ode_destroy": (None, [vp]),
        "mb_monodomain_desc_defaults": (None, [P(MbDesc)]),
        "mb_monodomain_create": (i32, [P(vp), P(MbDesc)]),
        "mb_monodomain_destroy": (None, [vp]),
        "mb_monodomain_step": (i32, [vp, i32]),
        "mb_monodomain_sync": (i32, [vp]),
        "mb_solve_all_volumes_odes": (i32, [vp]),
        "mb_update_monodomain_default": (i32, [vp]),
        "mb_conjugate_gradient": (i32, [vp, P(u32), P(dbl)]),
        "mb_advance_time": (i32, [vp]),
        "mb_monodomain_step_host": (i32, [vp, vp, vp]),
        "mb_monodomain_get_v": (i32, [vp, vp]),
        "mb_monodomain_get_activation": (i32, [vp, vp, vp, vp, vp]),
        "mb_monodomain_get_ecg": (i32, [vp, i64, i64, vp, vp, P(i64)]),
        "mb_monodomain_step_host_async": (i32, [vp, vp, vp]),
        "mb_monodomain_host_wait": (i32, [vp]),
        "mb_monodomain_time_steps_host_async": (i32, [vp, i32, vp, vp, vp, vp, P(dbl)]),
        "mb_batch_pack": (i32, [i32, vp, vp, P(i32), P(i32), vp, vp]),
        "mb_monodomain_checkpoint_bytes": (i32, [vp, P(C.c_size_t)]),
        "mb_monodomain_checkpoint": (i32, [vp, vp, C.c_size_t]),
        "mb_monodomain_restore": (i32, [vp, vp, C.c_size_t]),
        "mb_monodomain_save_v": (i32, [vp, C.c_char_p, i32]),
        "mb_adjoint_create": (i32, [P(vp), vp, i32, i32, i32, vp, i32]),
        "mb_adjoint_forward": (i32, [vp, vp, vp, vp]),
        "mb_adjoint_backward": (i32, [vp, vp, vp, vp]),
        "mb_adjoint_destroy": (None, [vp]),
        "mb_monodomain_set_v": (i32, [vp, vp]),
        "mb_monodomain_get_state": (i32, [vp, vp]),
        "mb_monodomain_info": (i32, [vp, P(i64), P(dbl), P(u32), P(i32)]),
        "mb_monodomain_step_stats": (i32, [vp, i64, i64, P(MbStepStats)]),
        "mb_monodomain_device_v": (i32, [vp, P(vp), P(vp)]),
        "mb_monodomain_profile_steps": (i32, [vp, i32, P(dbl), P(dbl), P(dbl), P(i32)]),
        "mb_csr_conjugate_gradient": (i32, [i32, vp, vp, vp, vp, vp, dbl, i32, i32, P(u32), P(dbl)]),
        "mb_csr_create": (i32, [P(vp), i32, vp, vp, vp]),
        "mb_csr_solve": (i32, [vp, vp, vp, dbl, i32, i32, P(u32), P(dbl)]),
        "mb_csr_destroy": (None, [vp]),
        "mb_monodomain_tuning": (i32, [vp, P(i32), P(i32), P(i32)]),
        "mb_cg_launch_shapes": (i32, [P(i32)]),
        "mb_monodomain_time_steps": (i32, [vp, i32, P(dbl)]),
        "mb_monodomain_time_steps_host": (i32, [vp, i32, vp, vp, P(dbl)]),
        "mb_csr_conjugate_gradient_noalloc": (i32, [i32, vp, vp, vp, vp, vp, dbl, i32, i32, P(u32), P(dbl), vp]),
        "mb_monodomain_save_state": (i32, [vp, C.c_char_p, i32]),
        "mb_monodomain_restore_state": (i32, [vp, C.c_char_p]),
        "mb_reference_cell_order": (i32, [i32, i32, i32, vp, vp, P(i64), P(i64)]),
        "mb_torord_endo_initial_state": (i32, [i32, P(dbl)]),
        "mb_torord_initial_state": (i32, [i32, P(dbl)]),
        "mb_ode_device_state": (i32, [vp, P(vp), P(C.c_size_t)]),
        "mb_ode_set_steps": (i32, [vp, dbl, C.c_uint32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


class _Lazy:
    """The library, loaded at its first use: importing the package (for
    the workload descriptions, say) maps no native code; the first call into
    the library loads it, and raises ImportError if it is missing."""

    _cdll = None

    def __getattr__(self, name):
        if _Lazy._cdll is None:
            _Lazy._cdll = _load()
        return getattr(_Lazy._cdll, name)


lib = _Lazy()


def check(rc: int) -> None:
    if rc != MB_OK:
        raise MonoAlgError(rc, lib.mb_last_error().decode(errors="replace"))


def device_count() -> int:
    n = C.c_int(0)
    check(lib.mb_device_count(C.byref(n)))
    return n.value
