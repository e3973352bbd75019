"""ctypes binding of libefs.so (include/efs.h).

Loading fails loudly: there is no CPU fallback behind this package.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libefs.so")

u32 = C.c_uint32
u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
szt = C.c_size_t
vp = C.c_void_p


class PmlRegion(C.Structure):
    _fields_ = [("start", u32 * 3), ("num", u32 * 3),
                ("vv", f32p), ("vvfo", f32p), ("vvfn", f32p),
                ("ii", f32p), ("iifo", f32p), ("iifn", f32p)]


class TfsfPoint(C.Structure):
    _fields_ = [("field_idx", u32), ("delay_int", u32), ("delay_frac", C.c_float), ("amp", C.c_float)]


class AdeDirection(C.Structure):
    _fields_ = [("dir", u32), ("pos_idx", u32p),
                ("v_int", f32p), ("v_ext", f32p), ("v_lor", f32p),
                ("i_int", f32p), ("i_ext", f32p), ("i_lor", f32p)]


class AdeOrder(C.Structure):
    _fields_ = [("num_cells", u32), ("has_lorentz", u32), ("num_directions", u32),
                ("directions", C.POINTER(AdeDirection))]


class RlcElement(C.Structure):
    _fields_ = [("field_idx", u32), ("direction", u32), ("type_flag", u32),
                ("i2v", C.c_float), ("ilv", C.c_float), ("vvd", C.c_float), ("vv2", C.c_float),
                ("vj1", C.c_float), ("vj2", C.c_float), ("ib0", C.c_float), ("b1", C.c_float), ("b2", C.c_float)]


# name -> (restype, argtypes)
SIGNATURES = {
    "efs_create": (C.c_int, [C.POINTER(vp), C.c_int]),
    "efs_destroy": (C.c_int, [vp]),
    "efs_last_error": (C.c_char_p, [vp]),
    "efs_init": (C.c_int, [vp, u32p, f32p, f32p, f32p, f32p]),
    "efs_init_indexed": (C.c_int, [vp, u32p, u32p, f32p, u32]),
    "efs_configure_excitation": (C.c_int, [vp, f32p, u32, u32p, f32p, u32p, u32p, u32, u32]),
    "efs_configure_pml": (C.c_int, [vp, u32, C.POINTER(PmlRegion)]),
    "efs_configure_mur": (C.c_int, [vp, f32p, u32p, u32p, u32]),
    "efs_configure_tfsf": (C.c_int, [vp, f32p, u32, u32, C.POINTER(TfsfPoint), u32, C.POINTER(TfsfPoint), u32]),
    "efs_configure_ade": (C.c_int, [vp, u32, C.POINTER(AdeOrder)]),
    "efs_configure_ade_apply": (C.c_int, [vp, C.c_int]),
    "efs_configure_rlc": (C.c_int, [vp, u32, C.POINTER(RlcElement)]),
    "efs_configure_pbc": (C.c_int, [vp, u32, u32p, f64p]),
    "efs_configure_steady_state": (C.c_int, [vp, u32p, u32, u32, C.c_float]),
    "efs_set_steady_state_recording": (C.c_int, [vp, C.c_int]),
    "efs_read_steady_state": (C.c_int, [vp, f32p, f32p, u32p, C.POINTER(C.c_int)]),
    "efs_iterate": (C.c_int, [vp, u32]),
    "efs_num_ts": (C.c_int, [vp, u32p]),
    "efs_sync": (C.c_int, [vp]),
    "efs_get_stream": (C.c_int, [vp, C.POINTER(vp)]),
    "efs_configure_probe_gather": (C.c_int, [vp, u32p, u32]),
    "efs_read_probe_gather": (C.c_int, [vp, f32p, szt]),
    "efs_configure_probe_gather_buffered": (C.c_int, [vp, u32p, u32, u32, u32]),
    "efs_read_probe_gather_buffered": (C.c_int, [vp, f32p, szt, u32p, u32p]),
    "efs_configure_nf2ff": (C.c_int, [vp, u32p, u32, f64p, u32, C.c_double, f32p, u32, u32]),
    "efs_read_nf2ff": (C.c_int, [vp, f32p, f32p, szt]),
    "efs_far_field": (C.c_int, [vp, u32, f32p, f32p, u32, f32p, u32, f64p, C.c_double, C.c_double, f32p]),
    "efs_far_field_time": (C.c_int, [vp, f32p]),
    "efs_energy": (C.c_int, [vp, C.c_int, f64p]),
    "efs_flush_energy": (C.c_int, [vp, f64p]),
    "efs_energy_noalloc": (C.c_int, [vp, f64p]),
    "efs_batch_create": (C.c_int, [C.POINTER(vp), C.POINTER(vp), C.c_uint32]),
    "efs_batch_destroy": (C.c_int, [vp]),
    "efs_batch_last_error": (C.c_char_p, [vp]),
    "efs_batch_iterate": (C.c_int, [vp, C.c_uint32]),
    "efs_batch_sync": (C.c_int, [vp]),
    "efs_batch_set_shape": (C.c_int, [vp, C.c_uint32, C.c_uint32]),
    "efs_batch_autotune": (C.c_int, [vp, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_float)]),
    "efs_get_fields": (C.c_int, [vp, f32p, f32p]),
    "efs_set_fields": (C.c_int, [vp, f32p, f32p]),
    "efs_get_planes": (C.c_int, [vp, u32, u32, vp, vp]),
    "efs_set_planes": (C.c_int, [vp, u32, u32, vp, vp]),
    "efs_get_state": (C.c_int, [vp, vp, szt, C.POINTER(szt)]),
    "efs_set_state": (C.c_int, [vp, vp, szt]),
    "efs_device_bytes": (C.c_int, [vp, C.POINTER(szt)]),
    "efs_debug_read": (C.c_int, [vp, C.c_char_p, u32, f32p, szt, C.POINTER(szt)]),
    "efs_time_core": (C.c_int, [vp, u32, f32p]),
    "efs_time_phases": (C.c_int, [vp, u32, f32p]),
    "efs_batch_time_phases": (C.c_int, [vp, u32, f32p]),
    "efs_debug_set_wait": (C.c_int, [vp, C.c_uint64, u32]),
    "efs_set_plane_depth": (C.c_int, [vp, u32]),
    "efs_kernels_per_step": (C.c_int, [vp, u32p]),
}

STATUS = {0: "EFS_OK", 1: "EFS_ERR_INVALID", 2: "EFS_ERR_STATE", 3: "EFS_ERR_CUDA",
          4: "EFS_ERR_OOM", 5: "EFS_ERR_TIMEOUT", 6: "EFS_ERR_RANGE"}

_lib = None


def load(path=LIB_PATH):
    """Load libefs.so and attach signatures.  Raises if it is missing."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libefs.so not built at %s: run efs_b200/build.py "
                          "(the engine has no CPU fallback)" % path)
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


class EfsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS.get(code, code), msg))
        self.code = code
