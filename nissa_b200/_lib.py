"""ctypes binding of libtmsolve.so (the C ABI declared in include/tmsolve.h)."""
from __future__ import annotations

import ctypes
import os

from . import build as _build

_lib = None

P = ctypes.c_void_p
D = ctypes.c_double
I = ctypes.c_int


class Stats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("iterations", ctypes.c_int32), ("reliable_updates", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("iterated_rel_res2", ctypes.c_double), ("true_rel_res2", ctypes.c_double),
                ("lx_rel_res2", ctypes.c_double), ("seconds", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


# name -> (restype, argtypes)
SIGNATURES = {
    "tms_create": (I, [ctypes.POINTER(P), I, I, D, I]),
    "tms_create4": (I, [ctypes.POINTER(P), I, I, I, I, D, I]),
    "tms_destroy": (I, [P]),
    "tms_last_error": (ctypes.c_char_p, [P]),
    "tms_set_pointer_mode": (I, [P, I]),
    "tms_volume": (ctypes.c_int64, [P]),
    "tms_geometry_tables": (I, [P, P, P, P, P, P]),
    "tms_conf_upload": (I, [P, P, I, I]),
    "tms_conf_is_su3": (I, [P]),
    "tms_clover_term": (I, [P, D]),
    "tms_clover_get": (I, [P, P]),
    "tms_tmclovDee": (I, [P, I, D, D, I, P, P]),
    "tms_inv_tmclovDee": (I, [P, D, D, I, P, P]),
    "tms_tmclovDkern_eoprec": (I, [P, D, I, D, D, I, P, P]),
    "tms_tmclovDkern_eoprec_square": (I, [P, D, I, D, D, P, P]),
    "tms_apply_tmclovQ": (I, [P, D, I, D, D, P, P]),
    "tms_cg_tmclov_eoprec_square": (I, [P, P, P, P, D, I, D, D, I, D, I, ctypes.POINTER(Stats)]),
    "tms_cg_tmclov_eoprec": (I, [P, P, P, D, I, D, D, D, I, D, I, ctypes.POINTER(Stats)]),
    "tms_rotate_twisted": (I, [P, I, P, P]),
    "tms_get_qprop": (I, [P, I, I, D, I, D, D, D, I, D, I, P, P, ctypes.POINTER(Stats)]),
    "tms_reconstruct_tm_doublet": (I, [P, D, I, D, D, P, P, P]),
    "tms_read_ildg": (I, [P, ctypes.c_char_p, P]),
    "tms_write_ildg": (I, [P, ctypes.c_char_p, P, I]),
    "tms_conf_load_ildg": (I, [P, ctypes.c_char_p, I]),
    "tms_conf_plaquette": (I, [P, I, ctypes.POINTER(D)]),
    "tms_hop_eo": (I, [P, I, P, P, I, D]),
    "tms_create_slab": (I, [ctypes.POINTER(P), I, I, I, I, I, I, D, I]),
    "tms_slab_face_sites": (ctypes.c_int64, [P]),
    "tms_slab_pack": (I, [P, I, P, P, P]),
    "tms_slab_hop": (I, [P, I, P, P, P, P, I, D]),
    "tms_slab_kern_half": (I, [P, I, D, D, P, P, P, P, P, I, D]),
    "tms_tmDee": (I, [P, D, D, P, P]),
    "tms_inv_tmDee": (I, [P, D, D, P, P]),
    "tms_kern_eoprec": (I, [P, D, I, D, D, P, P]),
    "tms_kern_eoprec_square": (I, [P, D, I, D, D, P, P]),
    "tms_apply_tmQ": (I, [P, D, I, D, D, P, P]),
    "tms_apply_tmQ2": (I, [P, D, I, D, D, P, P]),
    "tms_cg_eoprec_square": (I, [P, P, P, P, D, I, D, D, I, D, I, ctypes.POINTER(Stats)]),
    "tms_cg_eoprec": (I, [P, P, P, D, I, D, D, I, D, I, ctypes.POINTER(Stats)]),
    "tms_cg_eoprec_guess": (I, [P, P, P, P, D, I, D, D, I, D, I, ctypes.POINTER(Stats)]),
    "tms_cg_tmQ2": (I, [P, P, P, P, D, I, D, D, I, D, I, ctypes.POINTER(Stats)]),
    "tms_cgm_tmQ2": (I, [P, P, P, D, I, D, P, I, I, P, I, P]),
    "tms_cg_eoprec_batched": (I, [P, I, P, P, D, I, D, P, I, P, I, P]),
    "tms_cg_eoprec_columns": (I, [P, I, P, P, D, I, D, D, I, D, I, P]),
    "tms_batch_open": (I, [P, I, I, I, D, ctypes.POINTER(P)]),
    "tms_batch_submit": (I, [P, I, P, D, D, I, D]),
    "tms_batch_step": (I, [P, P, ctypes.POINTER(I)]),
    "tms_batch_collect": (I, [P, I, P, ctypes.POINTER(Stats)]),
    "tms_batch_close": (I, [P]),
    "tms_launch_count": (ctypes.c_uint64, [P]),
    "tms_hop_stage_timeouts": (ctypes.c_int64, [P]),
    "tms_set_tuning": (I, [P, ctypes.c_char_p, D]),
    "tms_get_tuning": (I, [P, ctypes.c_char_p, ctypes.POINTER(D)]),
    "tms_bench_hop": (I, [P, I, I, I, I, ctypes.POINTER(D), ctypes.POINTER(D)]),
    "tms_bench_hop_batched": (I, [P, I, I, I, I, ctypes.POINTER(D), ctypes.POINTER(D)]),
    "tms_hop_eo_noalloc": (I, [I, I, D, P, I, I, I, P, P, I, D, P, ctypes.c_char_p, I]),
}


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libtmsolve.so (building it first if it is missing or stale)."""
    global _lib
    if _lib is None:
        if build_if_missing and _build.stale():
            _build.build()
        if not os.path.exists(_build.LIB):
            raise RuntimeError("libtmsolve.so is not built (python -m nissa_b200.build)")
        L = ctypes.CDLL(_build.LIB)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
