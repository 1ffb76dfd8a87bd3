"""ctypes binding of the in-tree sm_100a library (viprs_b200/_lib/libviprs_b200.so).

The library is the product path: nothing here falls back to CPU code.  If the
shared object is missing, loading fails loudly with the build command to run.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libviprs_b200.so")

STATUS = {
    0: "ok", 1: "invalid argument", 2: "unsupported format or node", 3: "too many filter taps",
    4: "out of device memory", 5: "CUDA error", 6: "device wait timed out",
    7: "interpolation kernel not valid for this op", 8: "affine matrix determinant is singular",
    9: "null pointer", 10: "image size, bands or format mismatch",
    11: "work exceeds the static scratch of the no-alloc entry point",
}


class ViprsError(RuntimeError):
    """A non-zero viprs_status returned by the library."""

    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, 'status %d' % status)} (status {status})")


class Image(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("bands", ctypes.c_uint32), ("format", ctypes.c_int32), ("row_stride", ctypes.c_uint64)]


class Node(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("factor_u", ctypes.c_uint32), ("vfactor_u", ctypes.c_uint32),
                ("ceil_mode", ctypes.c_int32), ("factor", ctypes.c_double), ("vfactor", ctypes.c_double),
                ("kernel", ctypes.c_int32), ("matrix", ctypes.c_double * 4), ("tx", ctypes.c_double),
                ("ty", ctypes.c_double), ("out_width", ctypes.c_uint32), ("out_height", ctypes.c_uint32),
                ("extend", ctypes.c_int32), ("background", ctypes.c_double),
                ("premultiplied", ctypes.c_int32), ("area_x", ctypes.c_uint32), ("area_y", ctypes.c_uint32),
                ("area_width", ctypes.c_uint32), ("area_height", ctypes.c_uint32),
                ("demand_hint", ctypes.c_int32)]


_LIB = None

_P = ctypes.c_void_p
_I = ctypes.c_int32
_U = ctypes.c_uint32
_D = ctypes.c_double
_IMG = ctypes.POINTER(Image)

SIGNATURES = {
    "viprs_status_string": (ctypes.c_char_p, [_I]),
    "viprs_last_cuda_error": (_I, []),
    "viprs_sin_rn": (_I, [_P, _P, ctypes.c_int64]),
    "viprs_plan_status": (_I, [_P, _P]),
    "viprs_thumbnail_plan_nodes": (_I, [_I, _U, _U, _I, _I, _U, _U, _U, _I, _P, _I, ctypes.POINTER(_I),
                                       ctypes.POINTER(_U), ctypes.POINTER(_U), ctypes.POINTER(_U)]),
    "viprs_resize_plan_nodes": (_I, [_D, _D, _I, _D, _U, _U, _P, _I, ctypes.POINTER(_I), ctypes.POINTER(_U),
                                    ctypes.POINTER(_U)]),
    "viprs_reduce_output_len": (_U, [_D, _U]),
    "viprs_reduce_kernel_table": (_I, [_D, _I, ctypes.POINTER(_I), _P]),
    "viprs_reduceh": (_I, [_IMG, _IMG, _D, _I, _P]),
    "viprs_reducev": (_I, [_IMG, _IMG, _D, _I, _P]),
    "viprs_reduce": (_I, [_IMG, _IMG, _D, _D, _I, _P]),
    "viprs_shrinkh": (_I, [_IMG, _IMG, _U, _I, _P]),
    "viprs_shrinkv": (_I, [_IMG, _IMG, _U, _I, _P]),
    "viprs_shrink": (_I, [_IMG, _IMG, _U, _U, _P]),
    "viprs_zoom": (_I, [_IMG, _IMG, _U, _U, _P]),
    "viprs_similarity": (_I, [_IMG, _IMG, _D, _D, _I, _P]),
    "viprs_similarity_node": (_I, [_D, _D, _I, _U, _U, ctypes.POINTER(Node)]),
    "viprs_chain_output_size": (_I, [_U, _U, _P, _I, ctypes.POINTER(_U), ctypes.POINTER(_U)]),
    "viprs_premultiply": (_I, [_IMG, _IMG, _P]),
    "viprs_unpremultiply": (_I, [_IMG, _IMG, _P]),
    "viprs_affine": (_I, [_IMG, _IMG, ctypes.POINTER(_D), _D, _D, _I, _P]),
    "viprs_affine_backward_matrix": (_I, [_IMG, _IMG, ctypes.POINTER(_D), _D, _D, _I, _I, _D, _I, _U, _U, _P]),
    "viprs_mapim": (_I, [_IMG, _IMG, _IMG, _I, _I, _D, _I, _P]),
    "viprs_forward_affine_to_backward": (_I, [ctypes.POINTER(_D), _D, _D, ctypes.POINTER(_D),
                                              ctypes.POINTER(_D), ctypes.POINTER(_D)]),
    "viprs_chain_plan_create": (_I, [_U, _U, _U, _I, ctypes.POINTER(Node), _I, _I, ctypes.POINTER(_P)]),
    "viprs_thumbnail_plan_create": (_I, [_U, _U, _U, _I, _I, _U, _U, _I, _I, ctypes.POINTER(_P)]),
    "viprs_resize_plan_create": (_I, [_U, _U, _U, _I, _D, _D, _I, ctypes.POINTER(_P)]),
    "viprs_plan_output_size": (_I, [_P, ctypes.POINTER(_U), ctypes.POINTER(_U)]),
    "viprs_plan_workspace_bytes": (_I, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "viprs_plan_launch_count": (_I, [_P, ctypes.POINTER(_I)]),
    "viprs_plan_execute": (_I, [_P, _P, _P, _P]),
    "viprs_plan_execute_stages": (_I, [_P, _I, _I, _P, _P, _P]),
    "viprs_plan_execute_host": (_I, [_P, _P, _P, _P]),
    "viprs_plan_destroy": (None, [_P]),
    "viprs_thumbnail_batch_create": (_I, [_I, _P, _P, _P, _I, _U, _U, _I, _I, ctypes.POINTER(_P)]),
    "viprs_chain_batch_create": (_I, [_I, _P, _P, _P, _P, _I, _I, ctypes.POINTER(_P)]),
    "viprs_batch_output_size": (_I, [_P, _I, ctypes.POINTER(_U), ctypes.POINTER(_U)]),
    "viprs_batch_work_items": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "viprs_batch_launch_count": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "viprs_batch_execute": (_I, [_P, _P, _P, _P]),
    "viprs_batch_execute_graph": (_I, [_P, _P, _P, _P]),
    "viprs_batch_execute_per_image": (_I, [_P, _P, _P, _P]),
    "viprs_batch_autotune": (_I, [_P, _P, _P, _P, _I, ctypes.POINTER(ctypes.c_float)]),
    "viprs_batch_set_config": (_I, [_P, _U, _I, _I]),
    "viprs_batch_get_config": (_I, [_P, ctypes.POINTER(_U), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "viprs_batch_status": (_I, [_P, _P]),
    "viprs_batch_destroy": (None, [_P]),
    "viprs_reduce_noalloc": (_I, [_IMG, _IMG, _D, _D, _I, _P]),
    "viprs_reduce_adjoint": (_I, [_IMG, _IMG, _D, _I, _I, _P]),
    "viprs_reduce_hv_adjoint": (_I, [_IMG, _IMG, _D, _D, _I, _P]),
    "viprs_affine_grad": (_I, [_IMG, _IMG, _IMG, ctypes.POINTER(_D), _D, _D, _I, _I, _D, _I, _U, _U, _I, _P, _P]),
    "viprs_mapim_grad": (_I, [_IMG, _IMG, _IMG, _IMG, _IMG, _I, _I, _D, _I, _I, _P]),
}


def lib():
    """Load the library (once) and declare every exported signature."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing; build it with `python viprs_b200/build.py` "
                "(or __graft_entry__.build()). There is no CPU fallback.")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status, what):
    if status != 0:
        raise ViprsError(status, what)
