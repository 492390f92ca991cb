"""ctypes binding of the C ABI in include/rmt3d_gpu.h.

The library is the in-tree ``librmt3d_gpu.so``; importing this module fails
loudly when it is missing -- there is no CPU fallback for the FSI step.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librmt3d_gpu.so")

MAX_OBJ = 16
BLOCK_SHAPES = 5  # RMT3D_BLOCK_SHAPES
MAX_VEL_PROF = 8

OK = 0
REFMAP_UPDATE_ERR = 1
PROJECTION_ERR = 2
STEADY_SOLN_EXIT = 100
ERR_INVALID = -1
ERR_UNSUPPORTED = -2
ERR_CUDA = -3
ERR_EXTRAP = -4
ERR_NAN = -5
ERR_IO = -6
ERR_OOM = -7
ERR_TOO_LARGE = -8

SIM_FTEST, SIM_STEST, SIM_OBJECTS = 0, 1, 2
OBJ_BASIC_SPHERE, OBJ_SPHERE = 0, 1
FP64, MIXED, MIXED_BULK32 = 0, 1, 2


class ObjectDesc(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int),
        ("basic", ctypes.c_double * 4),
        ("extra", ctypes.c_double * 10),
        ("rho", ctypes.c_double),
        ("G", ctypes.c_double),
    ]


class RunDesc(ctypes.Structure):
    """rmt3d_run_desc: run controls and the restart point."""
    _fields_ = [
        ("suppress", ctypes.c_int), ("display", ctypes.c_int),
        ("chk_num", ctypes.c_int), ("chk_step", ctypes.c_int), ("chkpt_freq", ctypes.c_int),
        ("omp_num_thr", ctypes.c_int), ("debug_flag", ctypes.c_int), ("debug_obj_id", ctypes.c_int),
        ("obj_body", ctypes.c_int), ("data_fmt", ctypes.c_int), ("out_flag", ctypes.c_int),
        ("output_dim", ctypes.c_int), ("output_ind", ctypes.c_int),
        ("dump_code", ctypes.c_uint), ("ntracers", ctypes.c_int),
        ("current_time", ctypes.c_double),
        ("dirname", ctypes.c_char * 256), ("recover_dirname", ctypes.c_char * 256),
    ]


class SceneDesc(ctypes.Structure):
    _fields_ = [
        ("sys_size", ctypes.c_int * 3),
        ("bounds", ctypes.c_double * 6),
        ("periodic", ctypes.c_int * 3),
        ("bct", (ctypes.c_int * 6) * 3),
        ("bcv", (ctypes.c_double * 6) * 3),
        ("walls", ctypes.c_int * 6),
        ("wall_pos", ctypes.c_double * 6),
        ("wall_dist", ctypes.c_double),
        ("fmu", ctypes.c_double),
        ("frho", ctypes.c_double),
        ("fdt_pad", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("T", ctypes.c_double),
        ("frames", ctypes.c_int),
        ("stop_short", ctypes.c_int),
        ("num_iters", ctypes.c_int),
        ("sim_type", ctypes.c_int),
        ("has_exact", ctypes.c_int),
        ("godunov", ctypes.c_int),
        ("implicit_visc", ctypes.c_int),
        ("vel_prof_num", ctypes.c_int),
        ("vel_profile", ctypes.c_double * (2 * MAX_VEL_PROF)),
        ("n_obj", ctypes.c_int),
        ("nlayers", ctypes.c_int),
        ("max_extrap_rs", ctypes.c_int),
        ("wt_n", ctypes.c_double),
        ("ex_visc_mult", ctypes.c_double),
        ("ev_trans_mult", ctypes.c_double),
        ("sdt_pad", ctypes.c_double),
        ("dt_ex_pad", ctypes.c_double),
        ("weight_fac", ctypes.c_double),
        ("gravity", ctypes.c_double),
        ("obj", ObjectDesc * MAX_OBJ),
        ("var_den", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("mg_exact", ctypes.c_int),
        ("mixed_rtol", ctypes.c_double),
        ("run", RunDesc),
    ]


class MacroData(ctypes.Structure):
    """rmt3d_macro_data: one frame's macro.dat / centroid.dat values."""
    _fields_ = [
        ("time", ctypes.c_double), ("div_u_max", ctypes.c_double), ("div_u_min", ctypes.c_double),
        ("div_u_l2", ctypes.c_double), ("momentum", ctypes.c_double * 3),
        ("energy", ctypes.c_double), ("kinetic", ctypes.c_double), ("elastic", ctypes.c_double),
        ("potential", ctypes.c_double), ("power", ctypes.c_double),
        ("max_dev_detF", ctypes.c_double), ("dev_detF", ctypes.c_double),
        ("n_obj", ctypes.c_int),
        ("centroid", (ctypes.c_double * 3) * MAX_OBJ), ("velocity", (ctypes.c_double * 3) * MAX_OBJ),
    ]


class Request(ctypes.Structure):
    _fields_ = [("arrival_s", ctypes.c_double), ("steps", ctypes.c_int), ("desc", SceneDesc)]


class RequestResult(ctypes.Structure):
    _fields_ = [
        ("admit_s", ctypes.c_double), ("finish_s", ctypes.c_double), ("latency_s", ctypes.c_double),
        ("step_p50_ms", ctypes.c_double), ("step_p99_ms", ctypes.c_double),
        ("checksum", ctypes.c_double * 4), ("steps_done", ctypes.c_int), ("status", ctypes.c_int),
    ]


class ServeSummary(ctypes.Structure):
    _fields_ = [
        ("wall_s", ctypes.c_double), ("request_p50_s", ctypes.c_double), ("request_p99_s", ctypes.c_double),
        ("step_p50_ms", ctypes.c_double), ("step_p99_ms", ctypes.c_double),
        ("cellsteps_per_s", ctypes.c_double), ("requests", ctypes.c_int),
    ]


# entry points declared in include/rmt3d_gpu.h: name -> (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
SIGNATURES = {
    "rmt3d_desc_sizeof": (_I, []),
    "rmt3d_last_error": (ctypes.c_char_p, []),
    "rmt3d_desc_from_cfg": (_I, [ctypes.c_char_p, ctypes.POINTER(SceneDesc)]),
    "rmt3d_desc_defaults": (_I, [ctypes.POINTER(SceneDesc)]),
    "rmt3d_scene_create": (_I, [ctypes.POINTER(SceneDesc), _P, ctypes.POINTER(_P)]),
    "rmt3d_initialize": (_I, [_P]),
    "rmt3d_set_dt": (_I, [_P, _D]),
    "rmt3d_stepper_dt": (_I, [ctypes.POINTER(SceneDesc), _D, _DP, _IP]),
    "rmt3d_init_iter": (_I, [_P]),
    "rmt3d_write_chk_pt": (_I, [_P, _I, _I, ctypes.c_char_p, _I]),
    "rmt3d_read_chk_pt": (_I, [_P, ctypes.c_char_p, _IP]),
    "rmt3d_macro": (_I, [_P, ctypes.POINTER(MacroData)]),
    "rmt3d_tracer_positions": (_I, [_P, _P, _I, _IP]),
    "rmt3d_tracer_place": (_I, [_P, _P, _I]),
    "rmt3d_write_tracers": (_I, [_P, ctypes.c_char_p, _I]),
    "rmt3d_slice": (_I, [_P, _I, _I, _I, _I, _P, _IP, _IP]),
    "rmt3d_write_slice": (_I, [_P, _I, _I, _I, _I, _I, ctypes.c_char_p]),
    "rmt3d_prepare": (_I, [_P]),
    "rmt3d_step": (_I, [_P, _I, _IP]),
    "rmt3d_run": (_I, [_P, _I, _IP]),
    "rmt3d_step_phases": (_I, [_P, _I, _IP]),
    "rmt3d_get_scalar": (_I, [_P, _I, _DP]),
    "rmt3d_get_dims": (_I, [_P, _IP]),
    "rmt3d_get_field": (_I, [_P, _I, _P]),
    "rmt3d_get_refmap": (_I, [_P, _I, _P, _P, _P]),
    "rmt3d_import_reference": (_I, [_P, _P, _P, _P, _P, _I, _D, _D]),
    "rmt3d_export_reference": (_I, [_P, _P, _P, _P, _P, _I, _IP]),
    "rmt3d_diag": (_I, [_P, _I, _DP]),
    "rmt3d_sync": (_I, [_P]),
    "rmt3d_launch_count": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "rmt3d_scene_destroy": (_I, [_P]),
    "rmt3d_profile_kernel": (_I, [_P, _I, _I]),
    "rmt3d_profile_read": (_I, [_P, _DP, ctypes.POINTER(ctypes.c_longlong), _DP]),
    "rmt3d_batch_create": (_I, [ctypes.POINTER(SceneDesc), _I, _I, ctypes.POINTER(_P)]),
    "rmt3d_batch_prepare": (_I, [_P]),
    "rmt3d_batch_step": (_I, [_P, _I, _IP]),
    "rmt3d_batch_size": (_I, [_P, _IP]),
    "rmt3d_batch_scene": (_I, [_P, _I, ctypes.POINTER(_P)]),
    "rmt3d_batch_autotune": (_I, [_P, _I, _IP, _I, _IP]),
    "rmt3d_batch_set_smoother": (_I, [_P, _I]),
    "rmt3d_batch_destroy": (_I, [_P]),
    "rmt3d_scene_set_schedule": (_I, [_P, _I, _I, _I]),
    "rmt3d_scene_set_mg_launch": (_I, [_P, _I]),
    "rmt3d_scene_set_smoother": (_I, [_P, _I]),
    "rmt3d_scene_set_coarse_cluster": (_I, [_P, _I]),
    "rmt3d_scene_set_block_shape": (_I, [_P, _I]),
    "rmt3d_snapshot_fields": (_I, [_P, _IP, _I, ctypes.POINTER(_P)]),
    "rmt3d_snapshot_wait": (_I, [_P]),
    "rmt3d_scene_footprint": (ctypes.c_size_t, [ctypes.POINTER(SceneDesc)]),
    "rmt3d_scene_checksum": (_I, [_P, _DP]),
    "rmt3d_serve": (_I, [ctypes.POINTER(Request), _I, ctypes.c_size_t, _I,
                         ctypes.POINTER(RequestResult), ctypes.POINTER(ServeSummary)]),
    "rmt3d_serve_grouped": (_I, [ctypes.POINTER(Request), _I, ctypes.c_size_t, _I,
                                 ctypes.POINTER(RequestResult), ctypes.POINTER(ServeSummary)]),
    "rmt3d_div_u_noalloc": (_I, [_IP, _IP, _DP, _D, ctypes.POINTER(_P), ctypes.POINTER(_P), _P, _DP]),
}

_lib = None


def load():
    """Load the library (once) and attach the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "rmt3d_b200: CUDA library %s is missing; build it with "
            "`python -m rmt3d_b200.build` (there is no CPU fallback)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.rmt3d_desc_sizeof() != ctypes.sizeof(SceneDesc):
        raise ImportError("rmt3d_b200: descriptor size mismatch between ctypes and the library")
    _lib = lib
    return lib


class RMT3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("rmt3d error %d: %s" % (code, msg))
        self.code = code


def check(code):
    if code != OK:
        msg = _lib.rmt3d_last_error().decode() if _lib is not None else ""
        raise RMT3DError(code, msg)
    return code
