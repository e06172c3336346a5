"""ctypes binding of the C ABI declared in include/microcosmos_b200.h.

The shared library is built in-tree (``python -m microcosmos_b200.build``) and loaded
from this package directory.  There is no fallback: if the library is missing or a
call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmicrocosmos_b200.so")

MC_OK, MC_ERR_INVALID, MC_ERR_CUDA, MC_ERR_WORKSPACE, MC_ERR_UNSUPPORTED, MC_ERR_NOT_BOUND = range(6)
MC_FLAG_NONFINITE = 1
MC_FLAG_TIMEOUT = 2

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int32)


class McConfig(ctypes.Structure):
    _fields_ = [
        ("cycles_per_step", ctypes.c_int32),
        ("stiffness_stretch", ctypes.c_float),
        ("stiffness_shear", ctypes.c_float),
        ("damping", ctypes.c_float),
        ("enable_fluid", ctypes.c_int32),
        ("viscosity", ctypes.c_double),
        ("max_fluid_velocity", ctypes.c_double),
        ("ibm_iterations", ctypes.c_int32),
        ("synthetic_node_width", ctypes.c_float),
        ("ibm_kernel_size", ctypes.c_int32),
        ("ibm_relaxation", ctypes.c_float),
        ("node_mass", ctypes.c_float),
        ("lambda_trt", ctypes.c_float),
        ("enable_force_clamp", ctypes.c_int32),
        ("enable_steric", ctypes.c_int32),
        ("steric_strength", ctypes.c_float),
        ("steric_sigma", ctypes.c_double),
        ("steric_neighbor_skip", ctypes.c_int32),
        ("steric_scatter_value", ctypes.c_float),
        ("solver_type", ctypes.c_int32),
        ("solver_dt", ctypes.c_double),
    ]


class McDims(ctypes.Structure):
    _fields_ = [("H", ctypes.c_int32), ("W", ctypes.c_int32), ("N", ctypes.c_int32),
                ("E", ctypes.c_int32), ("B", ctypes.c_int32), ("fluid_H", ctypes.c_int32), ("fluid_W", ctypes.c_int32)]


class McState(ctypes.Structure):
    _fields_ = [
        ("position", ctypes.c_void_p),
        ("velocity", ctypes.c_void_p),
        ("theta", ctypes.c_void_p),
        ("rest_lengths", ctypes.c_void_p),
        ("bending_rest_angles", ctypes.c_void_p),
        ("bending_stiffness", ctypes.c_void_p),
        ("steric", ctypes.c_void_p),
        ("fluid_velocity", ctypes.c_void_p),
        ("f_grid", ctypes.c_void_p),
    ]


class McActuation(ctypes.Structure):
    _fields_ = [("c", ctypes.c_void_p), ("amp", ctypes.c_void_p), ("omega", ctypes.c_void_p),
                ("phase", ctypes.c_void_p), ("t0", ctypes.c_int32)]


class McRecord(ctypes.Structure):
    _fields_ = [("position", ctypes.c_void_p), ("velocity", ctypes.c_void_p), ("steric", ctypes.c_void_p),
                ("fluid_velocity", ctypes.c_void_p), ("every", ctypes.c_int32)]


class McStateCot(ctypes.Structure):
    _fields_ = [("position", ctypes.c_void_p), ("velocity", ctypes.c_void_p), ("theta", ctypes.c_void_p),
                ("f_grid", ctypes.c_void_p)]


class McParamGrads(ctypes.Structure):
    _fields_ = [("rest_angles", ctypes.c_void_p), ("act_c", ctypes.c_void_p), ("act_amp", ctypes.c_void_p),
                ("act_phase", ctypes.c_void_p), ("rest_lengths", ctypes.c_void_p),
                ("bending_stiffness", ctypes.c_void_p), ("act_omega", ctypes.c_void_p)]


class McEnv(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int32), ("E", ctypes.c_int32), ("B", ctypes.c_int32),
                ("H", ctypes.c_int32), ("W", ctypes.c_int32),
                ("base_rest_lengths", ctypes.c_void_p), ("base_bending_rest_angles", ctypes.c_void_p),
                ("d_rest_length", ctypes.c_void_p), ("d_bending_angle", ctypes.c_void_p),
                ("rest_lengths", ctypes.c_void_p), ("bending_rest_angles", ctypes.c_void_p),
                ("position", ctypes.c_void_p), ("velocity", ctypes.c_void_p),
                ("energy_center", ctypes.c_void_p), ("noise", ctypes.c_void_p),
                ("energy_walk_std", ctypes.c_float), ("energy_amplitude", ctypes.c_float),
                ("energy_two_size_sq", ctypes.c_float), ("max_steps", ctypes.c_int32),
                ("time", ctypes.c_void_p), ("done", ctypes.c_void_p),
                ("observation", ctypes.c_void_p), ("reward", ctypes.c_void_p),
                ("num_segments", ctypes.c_int32), ("segment_offsets", ctypes.c_void_p),
                ("segment_fitness", ctypes.c_void_p)]


# name -> (restype, argtypes); every symbol declared in include/microcosmos_b200.h
SIGNATURES = {
    "mc_plan_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(McDims), ctypes.POINTER(McConfig),
                                      c_float_p, ctypes.POINTER(c_int_p), ctypes.POINTER(c_int_p),
                                      ctypes.POINTER(ctypes.c_void_p)]),
    "mc_plan_destroy": (None, [ctypes.c_void_p]),
    "mc_plan_set_lbm_shape": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    "mc_plan_set_steric_method": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_steric_method": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_plan_set_fft_values_per_thread": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_fft_values_per_thread": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_plan_set_bin_threads": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_bin_threads": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_plan_set_bin_sort_capacity": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_bin_sort_capacity": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_plan_get_lbm_shape": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                             ctypes.POINTER(ctypes.c_int32)]),
    "mc_plan_set_lbm_staging": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_lbm_staging": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_plan_workspace_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "mc_plan_bind": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "mc_rollout": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(McState), ctypes.c_int32,
                                  ctypes.POINTER(ctypes.POINTER(McActuation)),
                                  ctypes.POINTER(ctypes.POINTER(McRecord)), ctypes.c_int32, ctypes.c_void_p]),
    "mc_rollout_begin": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(McState),
                                        ctypes.POINTER(ctypes.POINTER(McActuation)),
                                        ctypes.POINTER(ctypes.POINTER(McRecord)), ctypes.c_void_p]),
    "mc_rollout_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_void_p]),
    "mc_rollout_end": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mc_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(McState), ctypes.c_void_p]),
    "mc_plan_set_fused_ib": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_uses_fused_ib": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_plan_set_ib_cluster": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_ib_cluster": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_plan_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    "mc_plan_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_int64)]),
    "mc_plan_profile_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "mc_profile_kernel_names": (ctypes.c_char_p, []),
    "mc_plan_read_flags": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int32,
                                          ctypes.c_void_p]),
    "mc_plan_last_launch_count": (ctypes.c_int64, [ctypes.c_void_p]),
    "mc_steric_potential_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                   ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p]),
    "mc_grad_plan_create": (ctypes.c_int, [ctypes.POINTER(McDims), ctypes.POINTER(McConfig), ctypes.c_float,
                                           c_int_p, c_int_p, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    "mc_grad_plan_destroy": (None, [ctypes.c_void_p]),
    "mc_grad_plan_workspace_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "mc_grad_plan_checkpoint_every": (ctypes.c_int32, [ctypes.c_void_p]),
    "mc_grad_plan_bind": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]),
    "mc_grad_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(McState), ctypes.POINTER(McActuation),
                                       ctypes.c_void_p]),
    "mc_grad_backward": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(McStateCot), ctypes.POINTER(McStateCot),
                                        ctypes.POINTER(McParamGrads), ctypes.c_void_p]),
    "mc_env_table_bytes": (ctypes.c_size_t, [ctypes.c_int32]),
    "mc_env_table_upload": (ctypes.c_int, [ctypes.POINTER(McEnv), ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    "mc_env_act": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "mc_env_observe": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]),
    "mc_render_scratch_bytes": (ctypes.c_size_t, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "mc_render_frames": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p]),
    "mc_last_error": (ctypes.c_char_p, []),
    "mc_version": (ctypes.c_char_p, []),
}

_lib = None


class McError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"microcosmos_b200 error {status}: {msg}")
        self.status = status


def load(path: str | None = None):
    """Load (once) and return the shared library; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m microcosmos_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status):
    if status != MC_OK:
        msg = load().mc_last_error().decode()
        raise McError(status, msg)
