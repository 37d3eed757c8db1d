"""ctypes binding of libucg.so (include/ucg.h).

The shared library is the product: every numerical call goes through it.  If it
is missing or cannot be loaded the import fails loudly; there is no fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libucg.so")

UCG_OK = 0
UCG_E_BADARG = 1
UCG_E_CUDA = 2
UCG_E_OOM = 3
UCG_E_STEP_UNDERFLOW = 4
UCG_E_NONFINITE = 5
UCG_E_TIMEOUT = 6
UCG_E_STATE = 7
UCG_E_UNSUPPORTED = 8
UCG_E_NODEVICE = 9

UCG_OKADA_FP64 = 0
UCG_OKADA_REF32IO = 1
UCG_PREC_FP64 = 0
UCG_PREC_SPLIT_BF16 = 1
UCG_PREC_SPLIT_PAIR = 4
UCG_PREC_HMATRIX = 2
UCG_PREC_HMATRIX_SPLIT = 3
UCG_DRIVER_RATESTATE = 0
UCG_DRIVER_VISCOUSCYCLES = 1
UCG_ENS_STREAM_K = 0
UCG_ENS_SPLIT_LPT = 1
UCG_MLP_NIN = 11
UCG_MLP_NPARAM = 9153
UCG_MLP_NNORM = 24
UCG_TRACE_LEN = 14

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_long)
_vp = ctypes.c_void_p
_fp = ctypes.POINTER(ctypes.c_float)
_i = ctypes.c_int
_l = ctypes.c_long
_d = ctypes.c_double



class DeckInfo(ctypes.Structure):
    """ucg_deck_info"""
    _fields_ = [("driver", _i), ("lambda_", _d), ("mu", _d), ("interval", _d), ("n_rect", _i), ("n_tri", _i),
                ("n_vertex", _i), ("n_vol", _i), ("nonlinear_maxwell", _i), ("thermal", _i),
                ("n_obs_state", _i), ("n_obs_point", _i), ("n_events", _i)]


class RunOptions(ctypes.Structure):
    """ucg_run_options"""
    _fields_ = [("epsilon", _d), ("maximum_step", _d), ("maximum_iterations", _l), ("okada_mode", _i),
                ("precision", _i), ("device", _i), ("chunk", _l), ("wdir", ctypes.c_char_p), ("verbose", _i),
                ("hm_eta", _d), ("hm_eps", _d), ("hm_leaf", _i)]


# name -> (restype, argtypes); the complete exported surface of include/ucg.h
SIGNATURES = {
    "ucg_create": (_i, [ctypes.POINTER(_vp), _i, _d, _d, _i]),
    "ucg_destroy": (None, [_vp]),
    "ucg_strerror": (ctypes.c_char_p, [_i]),
    "ucg_last_error": (ctypes.c_char_p, [_vp]),
    "ucg_set_rectangles": (_i, [_vp, _i, _dp, _dp, _dp, _dp, _dp]),
    "ucg_set_triangles": (_i, [_vp, _i, _ip, _ip, _ip, _i, _dp]),
    "ucg_set_volumes": (_i, [_vp, _i, _dp, _dp, _dp, _dp, _dp]),
    "ucg_set_friction": (_i, [_vp] + [_dp] * 9),
    "ucg_set_rheology": (_i, [_vp, _dp, _dp, _dp, _i]),
    "ucg_assemble": (_i, [_vp, _i]),
    "ucg_assembly_times": (_i, [_vp, _dp, _dp, _dp]),
    "ucg_dims": (_i, [_vp, _lp, _lp]),
    "ucg_copy_G": (_i, [_vp, _dp, _l, _l, _l]),
    "ucg_set_precision": (_i, [_vp, _i]),
    "ucg_keep_fp64": (_i, [_vp, _i]),
    "ucg_build_hmatrix": (_i, [_vp, _i, _d, _d, _i]),
    "ucg_hmatrix_info": (_i, [_vp, _lp, _lp, _lp, _ip, _dp]),
    "ucg_hmatrix_matvec": (_i, [_vp, _dp, _dp]),
    "ucg_hmatrix_profile": (_i, [_vp, _i, _dp]),
    "ucg_state_len": (_l, [_vp]),
    "ucg_init_state": (_i, [_vp, _dp, _dp, _dp, _dp, _dp]),
    "ucg_odefun": (_i, [_vp, _d, _dp, _dp, _dp]),
    "ucg_set_tolerance": (_i, [_vp, _d, _d]),
    "ucg_rkqs": (_i, [_vp, _dp, _dp, _dp, _dp, _d, _dp, _dp, _lp]),
    "ucg_step": (_i, [_vp, _dp, _dp, _dp, _dp, _dp, _lp]),
    "ucg_set_state": (_i, [_vp, _dp, _d, _d]),
    "ucg_get_state": (_i, [_vp, _dp, _dp, _dp, _lp, _lp]),
    "ucg_run": (_i, [_vp, _d, _l, _lp]),
    "ucg_set_observation_points": (_i, [_vp, _i, _dp]),
    "ucg_build_O": (_i, [_vp, _i]),
    "ucg_observation_info": (_i, [_vp, _ip, _ip, _dp]),
    "ucg_copy_O": (_i, [_vp, _dp]),
    "ucg_displacements": (_i, [_vp, _dp, _dp, _dp, _dp]),
    "ucg_add_event": (_i, [_vp, _d, _dp]),
    "ucg_clear_events": (_i, [_vp]),
    "ucg_apply_perturbation": (_i, [_vp, _dp]),
    "ucg_record": (_i, [_vp, _i, _ip, _i, _l]),
    "ucg_record_len": (_l, [_vp]),
    "ucg_records": (_i, [_vp, _dp, _l, _lp, _lp]),
    "ucg_launch_count": (_l, [_vp]),
    "ucg_stream": (_vp, [_vp]),
    "ucg_profile_traction": (_i, [_vp, _i, _dp]),
    "ucg_test_wait_timeout": (_i, [_vp, _l, _i]),
    "ucg_odefun_noalloc": (_i, [_vp, _l, _l, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ucg_ens_create": (_i, [ctypes.POINTER(_vp), _i]),
    "ucg_ens_destroy": (None, [_vp]),
    "ucg_ens_last_error": (ctypes.c_char_p, [_vp]),
    "ucg_ens_add_geometry": (_i, [_vp, _vp, _i, _ip]),
    "ucg_ens_set_friction": (_i, [_vp, _i, _i] + [_dp] * 9),
    "ucg_ens_set_tolerance": (_i, [_vp, _d, _d]),
    "ucg_ens_set_state": (_i, [_vp, _i, _i, _d, _dp, _d]),
    "ucg_ens_get_state": (_i, [_vp, _i, _i, _dp, _dp, _dp, _lp, _lp, _ip]),
    "ucg_ens_set_states": (_i, [_vp, _i, _dp, _dp, _dp]),
    "ucg_ens_get_states": (_i, [_vp, _i, _dp, _dp, _dp, _lp, _lp, _ip]),
    "ucg_ens_put_states": (_i, [_vp, _i, _dp]),
    "ucg_ens_test_wait_timeout": (_i, [_vp, _l, _i]),
    "ucg_ens_set_increment_terms": (_i, [_vp, _i]),
    "ucg_ens_set_hier_planes": (_i, [_vp, _i]),
    "ucg_ens_plan": (_i, [_vp, _i, _i, _i]),
    "ucg_ens_tune": (_i, [_vp, _i, ctypes.c_char_p, _l]),
    "ucg_ens_use_graph": (_i, [_vp, _i]),
    "ucg_ens_run": (_i, [_vp, _d, _l, _lp]),
    "ucg_ens_matvec": (_i, [_vp, _i, _dp, _dp, _i]),
    "ucg_ens_set_event_threshold": (_i, [_vp, _d, _d]),
    "ucg_ens_get_events": (_i, [_vp, _i, _i, _lp, _dp]),
    "ucg_ens_info": (_i, [_vp, _lp, _ip, _lp, _lp, _lp, _dp, ctypes.c_char_p, _l]),
    "ucg_ens_stream": (_vp, [_vp]),
    "ucg_ens_profile_contract": (_i, [_vp, _i, _dp, _dp]),
    "ucg_mlp_create": (_i, [ctypes.POINTER(_vp), _i, ctypes.c_ulonglong]),
    "ucg_mlp_destroy": (None, [_vp]),
    "ucg_mlp_last_error": (ctypes.c_char_p, [_vp]),
    "ucg_mlp_set_params": (_i, [_vp, _fp, _fp]),
    "ucg_mlp_get_params": (_i, [_vp, _fp, _fp]),
    "ucg_mlp_set_data": (_i, [_vp, _fp, _fp, _l, _i]),
    "ucg_mlp_gradient": (_i, [_vp, _l, _l, _fp, _dp]),
    "ucg_mlp_train": (_i, [_vp, _i, _i, ctypes.c_float, ctypes.c_ulonglong, _fp]),
    "ucg_mlp_predict": (_i, [_vp, _fp, _l, _fp]),
    "ucg_ens_set_step_model": (_i, [_vp, _vp]),
    "ucg_ens_record_traces": (_i, [_vp, _l]),
    "ucg_ens_get_traces": (_i, [_vp, _fp, _l, _lp]),
    "ucg_deck_parse": (_i, [ctypes.c_char_p, _i, ctypes.POINTER(_vp), ctypes.c_char_p, _l]),
    "ucg_deck_read": (_i, [ctypes.c_char_p, _i, ctypes.POINTER(_vp), ctypes.c_char_p, _l]),
    "ucg_deck_free": (None, [_vp]),
    "ucg_deck_summary": (_i, [_vp, ctypes.POINTER(DeckInfo)]),
    "ucg_deck_wdir": (ctypes.c_char_p, [_vp]),
    "ucg_deck_point_name": (ctypes.c_char_p, [_vp, _i]),
    "ucg_deck_get": (_l, [_vp, ctypes.c_char_p, _dp, _l]),
    "ucg_deck_get_int": (_l, [_vp, ctypes.c_char_p, _ip, _l]),
    "ucg_deck_apply": (_i, [_vp, _vp]),
    "ucg_deck_create": (_i, [_vp, _i, ctypes.POINTER(_vp)]),
    "ucg_deck_init_state": (_i, [_vp, _vp, _dp]),
    "ucg_deck_run": (_i, [_vp, ctypes.POINTER(RunOptions), _lp, _dp]),
}

_lib = None


def load(path=LIB_PATH):
    """Load libucg.so and bind every entry point; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"libucg.so not found at {path}: build it with `python -m unicycle_b200.build` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class UcgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status
