"""ctypes binding of the C ABI in include/ep_gpu.h (``libepgpu.so``).

The library is built in-tree (``python -m ucla_cmg_b200.build``).  There is
no CPU fallback: if the library is missing or no CUDA device is usable,
every entry point raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libepgpu.so")

EP_OK = 0
ERRORS = {-1: "EP_ERR_ARG", -2: "EP_ERR_CUDA", -3: "EP_ERR_NOMEM", -4: "EP_ERR_MESH",
          -5: "EP_ERR_CG", -6: "EP_ERR_NEWTON", -7: "EP_ERR_NAN", -8: "EP_ERR_TIMEOUT",
          -9: "EP_ERR_UNSUPPORTED", -10: "EP_ERR_IO"}

LUORUDY, LUORUDYWITHGATE, TUSSCHER, MAHAJAN, MAHAJAN_FAIL = 0, 1, 2, 3, 4
PURKINJE = 5          # the Purkinje cell of .purk nodes (plugin level: ep_ionic_step)
FP64, FP32, SURROGATE = 0, 1, 2
TT_JAC_REFERENCE, TT_JAC_TRUE = 0, 1
SCHEME_CN, SCHEME_BE, SCHEME_EXPLICIT = 0, 1, 2

dp = C.POINTER(C.c_double)


class EPError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int32), ("xyz", dp), ("n_tets", C.c_int32),
                ("tets", C.POINTER(C.c_int32)), ("one_based", C.c_int32), ("fibers", dp),
                ("D", C.c_double * 3), ("Cm", C.c_double)]


class ModelDesc(C.Structure):
    _fields_ = [("model", C.c_int32), ("n_types", C.c_int32), ("type_consts", dp),
                ("node_type", C.POINTER(C.c_uint8)), ("node_gks_scale", dp),
                ("user_xi", C.c_double), ("newton_cap", C.c_int32), ("tt_jacobian", C.c_int32),
                ("mh_abs_mode", C.c_int32), ("initial_states", dp), ("newton_tol", C.c_double)]


class SolverDesc(C.Structure):
    _fields_ = [("dt", C.c_double), ("ionic_dt", C.c_double), ("cg_tol", C.c_double),
                ("cg_maxit", C.c_int32), ("smoothing_alpha", C.c_double),
                ("precision", C.c_int32), ("newton_tol", C.c_double), ("ecg_every", C.c_int32),
                ("act_threshold", C.c_double), ("scheme", C.c_int32), ("diffusion_dt", C.c_double)]


class StepStats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("cg_iters", C.c_int64), ("cg_max_iters", C.c_int32),
                ("cg_failures", C.c_int32), ("newton_iters", C.c_int64),
                ("newton_cap_hits", C.c_int32), ("nonfinite", C.c_int32),
                ("fallback_nodes", C.c_int64), ("device_ms", C.c_double), ("timeouts", C.c_int32),
                ("cg_ms", C.c_double), ("ionic_ms", C.c_double), ("ecg_ms", C.c_double),
                ("launches", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SurrogateDesc(C.Structure):
    _fields_ = [("n_in", C.c_int32), ("n_hidden", C.c_int32), ("n_hidden_layers", C.c_int32),
                ("n_out", C.c_int32), ("params", C.POINTER(C.c_float)),
                ("in_mean", C.POINTER(C.c_float)), ("in_std", C.POINTER(C.c_float)),
                ("out_mean", C.POINTER(C.c_float)), ("out_std", C.POINTER(C.c_float)),
                ("env_lo", C.POINTER(C.c_float)), ("env_hi", C.POINTER(C.c_float)),
                ("nah_max", C.c_float), ("log_mask", C.c_uint32),
                ("out_scale", C.POINTER(C.c_float)), ("out_lo", C.POINTER(C.c_float)),
                ("out_hi", C.POINTER(C.c_float)), ("hybrid_substeps", C.c_int32), ("v_update", C.c_int32)]


class CablesDesc(C.Structure):
    _fields_ = [("n_bars", C.c_int32), ("bars", C.POINTER(C.c_int32)), ("one_based", C.c_int32),
                ("fibers", dp), ("lv", C.POINTER(C.c_uint8)), ("Dp", C.c_double * 3),
                ("DpLeft", C.c_double * 3), ("radius", C.c_double), ("quad_order", C.c_int32),
                ("n_angle", C.c_int32), ("angle_nodes", C.POINTER(C.c_int32)), ("angle", dp),
                ("angle_sticky", C.c_int32), ("bar_angle", C.POINTER(C.c_int32))]


class LaunchConfig(C.Structure):
    _fields_ = [("cg_block", C.c_int32), ("cg_per_sm", C.c_int32), ("ionic_block", C.c_int32),
                ("graph_steps", C.c_int32), ("ionic_min_ctas", C.c_int32), ("cg_batch", C.c_int32),
                ("cg_variant", C.c_int32), ("cg_predict", C.c_int32),
                ("cg_prefetch", C.c_int32), ("sg_variant", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_L = None


def lib():
    """Load libepgpu.so (raises if it is not built)."""
    global _L
    if _L is not None:
        return _L
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built: run `python -m ucla_cmg_b200.build`")
    L = C.CDLL(LIB_PATH)
    H = C.c_void_p
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int32)
    sig = {
        "ep_version": ([], C.c_int),
        "ep_last_error": ([], C.c_char_p),
        "ep_model_nstate": ([C.c_int], C.c_int),
        "ep_model_nconst": ([C.c_int], C.c_int),
        "ep_model_default_consts": ([C.c_int, C.c_int, dp], C.c_int),
        "ep_create": ([C.POINTER(MeshDesc), C.POINTER(ModelDesc), C.POINTER(SolverDesc), C.c_int,
                       C.POINTER(H)], C.c_int),
        "ep_create_mixed": ([C.POINTER(MeshDesc), C.POINTER(CablesDesc), C.c_int32, C.POINTER(C.c_int32),
                             C.POINTER(ModelDesc), C.POINTER(SolverDesc), C.c_int, C.POINTER(H)], C.c_int),
        "ep_ecg_create": ([C.POINTER(MeshDesc), C.POINTER(CablesDesc), C.c_int32, dp, dp, C.c_int,
                           C.POINTER(H)], C.c_int),
        "ep_ecg_eval": ([H, C.c_int32, dp, dp], C.c_int),
        "ep_ecg_destroy": ([H], None),
        "ep_destroy": ([H], None),
        "ep_num_nodes": ([H], C.c_int),
        "ep_num_states": ([H], C.c_int),
        "ep_set_voltage": ([H, dp], C.c_int),
        "ep_get_voltage": ([H, dp], C.c_int),
        "ep_get_model_voltage": ([H, dp], C.c_int),
        "ep_get_states": ([H, dp], C.c_int),
        "ep_set_states": ([H, dp], C.c_int),
        "ep_set_stimulus": ([H, C.c_int32, C.POINTER(C.c_int32), dp, dp, dp], C.c_int),
        "ep_set_electrodes": ([H, C.c_int32, dp, dp], C.c_int),
        "ep_get_ecg": ([H, dp, C.c_int32, C.POINTER(C.c_int32), dp], C.c_int),
        "ep_compute_ecg": ([H, dp], C.c_int),
        "ep_step": ([H, C.c_int32, C.POINTER(StepStats)], C.c_int),
        "ep_get_time": ([H, dp, C.POINTER(C.c_int64)], C.c_int),
        "ep_set_profiling": ([H, C.c_int], C.c_int),
        "ep_diffusion_half_step": ([H, C.POINTER(C.c_int32), dp], C.c_int),
        "ep_cn_half_step_noalloc": ([C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                     C.c_int32, C.c_void_p, C.POINTER(C.c_int32), dp], C.c_int),
        "ep_get_activation": ([H, dp, dp], C.c_int),
        "ep_write_output": ([H, C.c_double, C.c_char_p], C.c_int),
        "ep_write_restart": ([H, C.c_double, C.c_char_p], C.c_int),
        "ep_read_restart": ([H, C.c_double, C.c_char_p], C.c_int),
        "ep_ionic_step": ([C.POINTER(ModelDesc), C.c_int32, C.c_int32, C.c_double, C.c_double,
                           dp, dp, dp, dp], C.c_int),
        "ep_ionic_phase": ([C.POINTER(ModelDesc), C.c_int32, C.c_int32, C.c_double, C.c_double,
                            C.c_double, dp, dp, dp], C.c_int),
        "ep_mlp_create": ([C.c_int32, C.POINTER(C.c_int32), C.c_uint64, C.c_int, C.POINTER(H)], C.c_int),
        "ep_mlp_destroy": ([H], None),
        "ep_mlp_num_params": ([H], C.c_int),
        "ep_mlp_get_params": ([H, fp], C.c_int),
        "ep_mlp_set_params": ([H, fp], C.c_int),
        "ep_mlp_forward": ([H, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p], C.c_int),
        "ep_mlp_loss_grad": ([H, C.c_void_p, C.c_void_p, fp, C.c_int32, dp, fp, C.c_void_p], C.c_int),
        "ep_mlp_adam_step": ([H, C.c_float, C.c_float, C.c_float, C.c_float], C.c_int),
        "ep_set_surrogate": ([H, C.POINTER(SurrogateDesc)], C.c_int),
        "ep_surrogate_forward": ([C.POINTER(SurrogateDesc), C.c_int32, fp, fp], C.c_int),
        "ep_batch_create": ([C.c_int32, C.POINTER(MeshDesc), C.POINTER(ModelDesc), C.POINTER(SolverDesc),
                             C.c_int, C.POINTER(H)], C.c_int),
        "ep_batch_layout": ([H, ip, ip, ip], C.c_int),
        "ep_batch_cg_last": ([H, ip, dp], C.c_int),
        "ep_batch_plan": ([C.c_int32, ip, C.c_int32, ip], C.c_int),
        "ep_assemble_operators": ([C.POINTER(MeshDesc), C.POINTER(CablesDesc), C.POINTER(SolverDesc),
                                   C.POINTER(C.c_int64), ip, ip, dp, dp, dp], C.c_int),
        "ep_get_launch_config": ([H, C.POINTER(LaunchConfig)], C.c_int),
        "ep_set_launch_config": ([H, C.POINTER(LaunchConfig)], C.c_int),
        "ep_autotune": ([H, C.c_int32, C.POINTER(LaunchConfig), dp, dp, ip], C.c_int),
        "ep_set_wait_limits": ([H, C.c_uint32, C.c_uint32], C.c_int),
        "ep_test_hold_barrier": ([H, C.c_int32], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _L = L
    return L


def exported_symbols():
    """Names declared in include/ep_gpu.h that the loaded library exports."""
    L = lib()
    out = []
    import re
    hdr = open(os.path.join(os.path.dirname(HERE), "include", "ep_gpu.h")).read()
    for name in sorted(set(re.findall(r"\b(ep_[a-z0-9_]+)\s*\(", hdr))):
        try:
            getattr(L, name)
            out.append((name, True))
        except AttributeError:
            out.append((name, False))
    return out


def check(rc):
    if rc != EP_OK:
        raise EPError(rc, lib().ep_last_error().decode(errors="replace"))
    return rc


def ptr(a, t=dp):
    return None if a is None else a.ctypes.data_as(t)


def model_nstate(model):
    return lib().ep_model_nstate(model)


def default_consts(model, ctype=0):
    nc = lib().ep_model_nconst(model)
    out = np.zeros(nc)
    check(lib().ep_model_default_consts(model, ctype, ptr(out)))
    return out
