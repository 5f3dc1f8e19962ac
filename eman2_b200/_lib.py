"""ctypes binding of libeman2_b200.so (the C ABI in include/eman2_b200.h).

The shared library is built in-tree (``python -m eman2_b200.build``).  There is
no CPU fallback: importing the binding without the library, or calling it
without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes
import os

from .exceptions import raise_status

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeman2_b200.so")

FR_OK = 0
MODE_IDS = {"nearest_neighbor": 1, "gauss_2": 2, "gauss_5": 5, "trilinear": 6}
MODE_ITER = 7   # FourierIterReconstructor's inserter
SCHED = {"auto": 0, "scatter": 1, "gather": 2}

_P = ctypes.c_void_p
_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int)


class fr_params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("mode", ctypes.c_int), ("sym", ctypes.c_char * 16), ("corners", ctypes.c_int),
                ("sqrtnorm", ctypes.c_int), ("usessnr", ctypes.c_int), ("verbose", ctypes.c_int)]


class fr_particle(ctypes.Structure):
    _fields_ = [("rot", ctypes.c_float * 9), ("tx", ctypes.c_float), ("ty", ctypes.c_float),
                ("weight", ctypes.c_float), ("defocus", ctypes.c_float),
                ("dfdiff", ctypes.c_float), ("dfang", ctypes.c_float),
                ("voltage", ctypes.c_float), ("cs", ctypes.c_float), ("apix", ctypes.c_float),
                ("ampcont", ctypes.c_float)]


class fr_stats(ctypes.Structure):
    _fields_ = [("kernel_launches", ctypes.c_longlong), ("insert_launches", ctypes.c_longlong),
                ("slices_inserted", ctypes.c_longlong), ("insert_ms", ctypes.c_double),
                ("gather_ms", ctypes.c_double), ("gather_launches", ctypes.c_longlong)]


# Every entry point the header declares, with its argument types.
SIGNATURES = {
    "fr_create": ([ctypes.POINTER(fr_params), ctypes.POINTER(_P)], ctypes.c_int),
    "fr_destroy": ([_P], ctypes.c_int),
    "fr_set_stream": ([_P, _P], ctypes.c_int),
    "fr_get_stream": ([_P, _P], ctypes.c_int),
    "fr_setup": ([_P], ctypes.c_int),
    "fr_setup_seed": ([_P, _P, ctypes.c_float], ctypes.c_int),
    "fr_setup_seedandweights": ([_P, _P, _P], ctypes.c_int),
    "fr_clear": ([_P], ctypes.c_int),
    "fr_preprocess_slices": ([_P, _P, ctypes.c_int, _P, _P], ctypes.c_int),
    "fr_insert_slices": ([_P, _P, ctypes.c_int, _P, _P, _P, ctypes.c_int, _I, ctypes.c_int],
                         ctypes.c_int),
    "fr_insert_particles": ([_P, _P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int], ctypes.c_int),
    "fr_determine_slice_agreement": ([_P, _P, ctypes.c_int, _P, _P, ctypes.c_float, ctypes.c_int,
                                      _P], ctypes.c_int),
    "fr_projection": ([_P, _P, _P], ctypes.c_int),
    "fr_projection_xf": ([_P, _P, ctypes.c_int, _P], ctypes.c_int),
    "fr_finish": ([_P, ctypes.c_int, _P, _P], ctypes.c_int),
    "fr_finish_async": ([_P, ctypes.c_int, _P, _P, _P], ctypes.c_int),
    "fr_get_accumulators": ([_P, _P, _P], ctypes.c_int),
    "fr_get_size": ([_P, _I], ctypes.c_int),
    "fr_footprint_bytes": ([ctypes.c_int], ctypes.c_size_t),
    "fr_sym_ops": ([ctypes.c_char_p, _F, ctypes.c_int], ctypes.c_int),
    "fr_last_error": ([], ctypes.c_char_p),
    "fr_profile": ([ctypes.c_int], ctypes.c_int),
    "fr_stats_get": ([ctypes.POINTER(fr_stats)], ctypes.c_int),
    "fr_stats_reset": ([], ctypes.c_int),
    "fr_version": ([], ctypes.c_char_p),
    "fr_batch_create": ([ctypes.POINTER(fr_params), ctypes.c_int, ctypes.POINTER(_P)],
                        ctypes.c_int),
    "fr_batch_destroy": ([_P], ctypes.c_int),
    "fr_batch_set_stream": ([_P, _P], ctypes.c_int),
    "fr_batch_insert_particles": ([_P, ctypes.POINTER(_P), _I, _I, ctypes.POINTER(_P)],
                                  ctypes.c_int),
    "fr_batch_finish": ([_P, ctypes.c_int, ctypes.c_int, _P, _P], ctypes.c_int),
    "fr_insert_particles_multi": ([ctypes.POINTER(_P), ctypes.c_int, ctypes.POINTER(_P), _I, _I,
                                   ctypes.POINTER(_P), _P], ctypes.c_int),
    "fr_batch_get_accumulators": ([_P, ctypes.c_int, _P, _P], ctypes.c_int),
    "fr_autotune": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _I, _F],
                    ctypes.c_int),
    "fr_set_tile": ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "fr_update_peaks": ([_P, _P, _P], ctypes.c_int),
    "fr_set_wiener": ([_P, ctypes.c_int], ctypes.c_int),
    "fr_set_reference": ([_P, _P, ctypes.c_int], ctypes.c_int),
    "fr_insert_slices_wiener": ([_P, _P, ctypes.c_int, _P, _P, _P, ctypes.c_int, _P, _P],
                                ctypes.c_int),
    "fr_decode_images": ([_P, ctypes.c_int, ctypes.c_int, ctypes.c_longlong, _P, _P], ctypes.c_int),
    "fr_finish_corrected": ([_P, ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P],
                            ctypes.c_int),
    "fr_kernel_fix": ([_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, _P],
                      ctypes.c_int),
    "fr_batch_graph_create": ([_P, _P, _P, _P, _P], ctypes.c_int),
    "fr_graph_create": ([_P, ctypes.c_int, _P, _P, _P, _P, _P], ctypes.c_int),
    "fr_graph_slot": ([_P, ctypes.c_int, _P], ctypes.c_int),
    "fr_graph_launch": ([_P, _P, _P], ctypes.c_int),
    "fr_graph_destroy": ([_P], ctypes.c_int),
    "fr_insert_slices_noalloc": ([_P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                  _P, _P, _P, _P, _P], ctypes.c_int),
}

_lib = None


def load():
    """Load the library (once).  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m eman2_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(rc: int) -> int:
    if rc != FR_OK:
        raise_status(rc, load().fr_last_error().decode(errors="replace"))
    return rc


def ptr(a) -> int:
    """Raw address of a contiguous numpy array or torch tensor (host or CUDA)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def stats() -> dict:
    st = fr_stats()
    check(load().fr_stats_get(ctypes.byref(st)))
    return {k: getattr(st, k) for k, _ in fr_stats._fields_}
