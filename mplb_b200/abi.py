"""ctypes mirror of include/mplbgpu.h and the loader of the native library.

The product path is the CUDA library ``libmplbgpu.so`` built next to this
file; there is no Python or CPU fallback for the stream-collision step, so a
missing or unloadable library raises ``NativeLibraryError``.
"""
import ctypes
import os

ABI_VERSION = 3

OK = 0
ERR_INVALID = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_DIVERGED = 4
ERR_TIMEOUT = 5
ERR_NO_DEVICE = 6
ERR_STATE = 7
STATUS_NAMES = {
    OK: "OK", ERR_INVALID: "INVALID", ERR_UNSUPPORTED: "UNSUPPORTED",
    ERR_CUDA: "CUDA", ERR_DIVERGED: "DIVERGED", ERR_TIMEOUT: "TIMEOUT",
    ERR_NO_DEVICE: "NO_DEVICE", ERR_STATE: "STATE",
}

# BoundarySurface (Src/boundary_host_device.h:7-29)
SURFACES = {
    "Left": 0, "Right": 1, "Top": 2, "Bottom": 3, "Front": 4, "Back": 5,
    "LeftBack": 50, "LeftFront": 40, "RightBack": 51, "RightFront": 41,
    "TopBack": 52, "TopFront": 42, "BottomBack": 53, "BottomFront": 43,
    "LeftTop": 20, "LeftBottom": 30, "RightTop": 21, "RightBottom": 31,
}
# VertexType (Src/flowfield_host_device.h:21-37)
VERTEX_TYPES = {
    "Fluid": 10, "Inlet": 11, "OutLet": 12, "MDPeriodic": 13, "Symmetry": 14,
    "FDPeriodic": 15, "Wall": 1000, "ImmersedSolid": -1,
    "ImmersedBoundary": -2, "VirtualBoundary": -3,
}
# BoundaryScheme (Src/boundary.h:70-83) + this path's halfway bounce-back.
# "EQMDiffuseREfl" is the reference's own JSON spelling
# (Src/configuration.cpp:86).
BC_SCHEMES = {
    "KineticDiffuseWall": 11, "KineticSpelluarWall": 12,
    "ExtrapolPressure1ST": 16, "ExtrapolPressure2ND": 17, "MDPeriodic": 18,
    "FDPeriodic": 19, "BounceBack": 20, "FreeFlux": 21, "ZouHeVelocity": 22,
    "EQNNoSlip": 23, "EQMDiffuseRefl": 24, "EQMDiffuseREfl": 24, "None": -1,
    "HalfwayBounceBack": 100,
}
D2Q9 = 9
D3Q19 = 19
FP64 = 0
FP32_SHIFTED = 1
FP16_SHIFTED = 2
PRECISIONS = {"fp64": FP64, "fp32": FP32_SHIFTED, "fp16": FP16_SHIFTED}
FORCE_NONE = 0
FORCE_1ST = 1
# SchemeType (Src/scheme.h:67-72)
SCHEME_STREAM_COLLISION = 10
SCHEME_STREAM_COLLISION_SWAP = 11
SCHEMES = {"Scheme_StreamCollision": SCHEME_STREAM_COLLISION,
           "Scheme_StreamCollision_Swap": SCHEME_STREAM_COLLISION_SWAP}


class Block(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int), ("size", ctypes.c_int * 3),
                ("cut", ctypes.c_int)]


class Connection(ctypes.Structure):
    _fields_ = [("from_block", ctypes.c_int), ("from_surface", ctypes.c_int),
                ("to_block", ctypes.c_int), ("to_surface", ctypes.c_int),
                ("type", ctypes.c_int)]


class Boundary(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int), ("surface", ctypes.c_int),
                ("scheme", ctypes.c_int), ("vertex_type", ctypes.c_int),
                ("given", ctypes.c_double * 3)]


class Desc(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int), ("space_dim", ctypes.c_int),
        ("lattice", ctypes.c_int), ("precision", ctypes.c_int),
        ("nblocks", ctypes.c_int), ("blocks", ctypes.POINTER(Block)),
        ("nconnections", ctypes.c_int),
        ("connections", ctypes.POINTER(Connection)),
        ("nboundaries", ctypes.c_int),
        ("boundaries", ctypes.POINTER(Boundary)),
        ("tau_ref", ctypes.c_double), ("dt", ctypes.c_double),
        ("cs", ctypes.c_double), ("body_force", ctypes.c_int),
        ("accel", ctypes.c_double * 3), ("force_velocity", ctypes.c_int),
        ("scheme", ctypes.c_int),
    ]


class Cavity(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("lid_u", ctypes.c_double),
                ("tau_ref", ctypes.c_double)]


class BatchTuning(ctypes.Structure):
    _fields_ = [("tile_nodes", ctypes.c_int), ("persistent", ctypes.c_int),
                ("chunk", ctypes.c_int), ("ctas_per_sm", ctypes.c_int)]


class NativeLibraryError(RuntimeError):
    """The CUDA library is missing or failed to load."""


PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(PACKAGE_DIR, "libmplbgpu.so")

_lib = None

_SIGNATURES = {
    "mplbgpu_create": (ctypes.c_int, [ctypes.POINTER(Desc),
                                      ctypes.POINTER(ctypes.c_void_p)]),
    "mplbgpu_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "mplbgpu_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "mplbgpu_init_macro": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] +
                           [ctypes.c_void_p] * 4),
    "mplbgpu_upload_f": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p]),
    "mplbgpu_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mplbgpu_update_macro": (ctypes.c_int, [ctypes.c_void_p]),
    "mplbgpu_residual": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p]),
    "mplbgpu_download_macro": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] +
                               [ctypes.c_void_p] * 4),
    "mplbgpu_download_f": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p]),
    "mplbgpu_mass": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mplbgpu_face_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "mplbgpu_export_face": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_void_p]),
    "mplbgpu_import_face": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_void_p]),
    "mplbgpu_residual_sums": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p]),
    "mplbgpu_check_health": (ctypes.c_int, [ctypes.c_void_p]),
    "mplbgpu_step_begin": (ctypes.c_int, [ctypes.c_void_p]),
    "mplbgpu_step_finish": (ctypes.c_int, [ctypes.c_void_p]),
    "mplbgpu_get_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mplbgpu_step_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int)]),
    "mplbgpu_set_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "mplbgpu_boundary_extent": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_void_p]),
    "mplbgpu_set_boundary_velocity": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p]),
    "mplbgpu_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "mplbgpu_launch_count": (ctypes.c_longlong, [ctypes.c_void_p]),
    "mplbgpu_last_step_ms": (ctypes.c_int, [ctypes.c_void_p,
                                            ctypes.c_void_p]),
    "mplbgpu_batch_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                            ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "mplbgpu_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "mplbgpu_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "mplbgpu_batch_set_tuning": (ctypes.c_int, [ctypes.c_void_p,
                                                ctypes.c_void_p]),
    "mplbgpu_batch_set_wait_limit": (ctypes.c_int, [ctypes.c_void_p,
                                                    ctypes.c_longlong]),
    "mplbgpu_batch_get_tuning": (ctypes.c_int, [ctypes.c_void_p,
                                                ctypes.c_void_p]),
    "mplbgpu_batch_init": (ctypes.c_int, [ctypes.c_void_p] +
                           [ctypes.c_void_p] * 3),
    "mplbgpu_batch_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mplbgpu_batch_run": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_double,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "mplbgpu_batch_download_macro": (ctypes.c_int, [ctypes.c_void_p] +
                                     [ctypes.c_void_p] * 3),
    "mplbgpu_batch_stats": (ctypes.c_int, [ctypes.c_void_p] +
                            [ctypes.c_void_p] * 3),
    "mplbgpu_residual_sums_noalloc": (ctypes.c_int, [
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong,
        ctypes.c_void_p, ctypes.c_void_p]),
}
NOALLOC_MAX_NODES = 16777216


# ---- include/mplbnn.h (warm-start network) ----
NN_GRID = 128


class NNView(ctypes.Structure):
    _fields_ = [("ptr", ctypes.c_void_p), ("nimg", ctypes.c_int),
                ("h", ctypes.c_int), ("w", ctypes.c_int), ("c", ctypes.c_int),
                ("ps", ctypes.c_longlong)]


_vp, _ip, _fp, _dp = (ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
                      ctypes.c_double)
_llp = ctypes.POINTER(ctypes.c_longlong)
_SIGNATURES.update({
    "mplbnn_conv_forward": (_ip, [ctypes.POINTER(NNView), _vp, _ip, _vp, _ip,
                                  ctypes.POINTER(NNView), _ip,
                                  ctypes.POINTER(NNView), _vp]),
    "mplbnn_conv_wgrad": (_ip, [ctypes.POINTER(NNView),
                                ctypes.POINTER(NNView), _ip, _vp, _vp]),
    "mplbnn_error": (ctypes.c_char_p, []),
    "mplbnn_create": (_ip, [_ip, ctypes.POINTER(_vp)]),
    "mplbnn_destroy": (_ip, [_vp]),
    "mplbnn_last_error": (ctypes.c_char_p, [_vp]),
    "mplbnn_synchronize": (_ip, [_vp]),
    "mplbnn_param_count": (ctypes.c_longlong, [_vp]),
    "mplbnn_layer_count": (_ip, []),
    "mplbnn_layer_info": (_ip, [_ip, ctypes.POINTER(_ip), ctypes.POINTER(_ip),
                                ctypes.POINTER(_ip), _llp, _llp]),
    "mplbnn_init_params": (_ip, [_vp, ctypes.c_ulonglong]),
    "mplbnn_set_params": (_ip, [_vp, _vp]),
    "mplbnn_get_params": (_ip, [_vp, _vp]),
    "mplbnn_get_grads": (_ip, [_vp, _vp]),
    "mplbnn_forward": (_ip, [_vp, _vp, _ip, _vp]),
    "mplbnn_loss_grad": (_ip, [_vp, _vp, _vp, _vp, _ip, ctypes.POINTER(_dp)]),
    "mplbnn_adam_step": (_ip, [_vp, _fp, _fp, _fp, _fp]),
    "mplbnn_fields_to_grid": (_ip, [_vp, _vp, _vp, _vp, _ip, _vp, _vp, _vp,
                                    _vp, _vp]),
    "mplbnn_grid_to_fields": (_ip, [_vp, _vp, _ip, _vp, _vp, _vp, _vp, _vp,
                                    _vp, _vp]),
})


def exported_symbols():
    """Names every build of the library must export (from mplbgpu.h and
    mplbnn.h)."""
    return sorted(_SIGNATURES)


def load_library(path=None):
    """Loads libmplbgpu.so (fails loudly; there is no fallback path)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIBRARY_PATH
    if not os.path.exists(p):
        raise NativeLibraryError(
            f"{p} is missing: build it with `python -m mplb_b200.build` "
            "(nvcc, sm_100a)")
    try:
        lib = ctypes.CDLL(p)
    except OSError as exc:
        raise NativeLibraryError(f"cannot load {p}: {exc}") from exc
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
