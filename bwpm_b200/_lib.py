"""ctypes binding of libbwpm_b200.so (the C ABI declared in include/bwpm_b200.h).

The library is built in-tree (make -C bwpm_b200/csrc, or __graft_entry__.build()). There is no
fallback: importing this module without the library raises ImportError.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("BWPM_B200_LIB", Path(__file__).resolve().parent / "libbwpm_b200.so"))

BWPM_OK, BWPM_EINVAL, BWPM_ERUNTIME = 0, 1, 2

if not LIB_PATH.exists():
    raise ImportError(
        f"{LIB_PATH} is missing: build the CUDA core first (make -C bwpm_b200/csrc); "
        "bwpm_b200 has no CPU fallback")

lib = ctypes.CDLL(str(LIB_PATH))

_d = ctypes.c_double
_sz = ctypes.c_size_t
_i = ctypes.c_int
_p = ctypes.c_void_p
_i64p = ctypes.POINTER(ctypes.c_int64)

# Signatures: (name, restype, argtypes). Every name here is declared in include/bwpm_b200.h.
SIGNATURES: dict[str, tuple] = {
    "bwpm_last_error": (_sz, [ctypes.c_char_p, _sz]),
    "bwpm_version": (ctypes.c_char_p, []),
    "bwpm_cuda_device_count": (_i, []),
    "bwpm_interface_matrices": (_i, [_i, _p, _p, _sz, _d, _d, _d, _d, _d, _p]),
    "bwpm_longitudinal_wavenumber": (_i, [_d, _d, _d, _p, _sz, _p]),
    "bwpm_solver_create": (_i, [_sz, _sz, _d, _d, _d, _d, _p, _sz, _p, _sz, _d, _d, _p, _i, _p,
                                _i, _d, ctypes.POINTER(_p)]),
    "bwpm_solver_create_geometry": (_i, [_sz, _sz, _d, _d, _d, _d, _p, _sz, _i, _p, _sz, _sz, _d,
                                         _d, _p, _i, _i, ctypes.POINTER(_p)]),
    "bwpm_geometry_labels": (_i, [_i, _i, _p, _sz, _sz, _sz, _sz, _d, _d, _d, _p]),
    "bwpm_solver_run": (_i, [_p, _p, _i, _p, _sz, _p, _p, _p, _p, _p, _p, _i64p]),
    "bwpm_solver_stats": (_i, [_p, _i64p, _i64p, _i64p]),
    "bwpm_solver_destroy": (None, [_p]),
    "bwpm_batch_create": (_i, [_i, ctypes.POINTER(_p)]),
    "bwpm_batch_add": (_i, [_p, _sz, _d, _d, _d, _p, _sz, _p, _sz, _d, _d, _p, _p, _i, _i64p]),
    "bwpm_batch_set_autotune": (_i, [_p, _i]),
    "bwpm_batch_set_variant": (_i, [_p, _sz, _i]),
    "bwpm_batch_class_info": (_i, [_p, ctypes.c_int64, _i64p, _i64p, _i64p, _i64p, _i64p,
                                   ctypes.POINTER(ctypes.c_float)]),
    "bwpm_variant_count": (_i, [_sz]),
    "bwpm_batch_prepare": (_i, [_p]),
    "bwpm_batch_run": (_i, [_p, ctypes.POINTER(ctypes.c_float)]),
    "bwpm_batch_solve_packed": (_i, [_p, _p, _p, ctypes.POINTER(ctypes.c_float)]),
    "bwpm_batch_result": (_i, [_p, ctypes.c_int64, _p, _p, _p, _p, _p, _p]),
    "bwpm_batch_stats": (_i, [_p, _i64p, _i64p, _i64p, _i64p, _i64p]),
    "bwpm_batch_work": (_i, [_p, ctypes.POINTER(_d), ctypes.POINTER(_d), ctypes.POINTER(_d)]),
    "bwpm_batch_destroy": (None, [_p]),
    "bwpm_server_create": (_i, [_i, ctypes.c_uint64, _i, _i, _i, ctypes.POINTER(_p)]),
    "bwpm_server_submit_2d": (_i, [_p, _sz, _d, _d, _d, _p, _sz, _p, _sz, _d, _d, _p, _p, _i,
                                   _i64p]),
    "bwpm_server_submit_3d": (_i, [_p, _sz, _sz, _d, _d, _d, _d, _p, _sz, _p, _sz, _d, _d, _p, _p,
                                   _i, _i64p]),
    "bwpm_server_submit_2d_borrowed": (_i, [_p, _sz, _d, _d, _d, _p, _sz, _p, _sz, _d, _d, _p, _p,
                                            _i, _i64p]),
    "bwpm_server_submit_3d_borrowed": (_i, [_p, _sz, _sz, _d, _d, _d, _d, _p, _sz, _p, _sz, _d, _d,
                                            _p, _p, _i, _i64p]),
    "bwpm_server_submit_3d_geometry": (_i, [_p, _sz, _sz, _d, _d, _d, _d, _p, _sz, _i, _p, _sz,
                                            _sz, _d, _d, _p, _p, _i, _i64p]),
    "bwpm_server_wait": (_i, [_p, ctypes.c_int64, _d, ctypes.POINTER(_i)]),
    "bwpm_server_result": (_i, [_p, ctypes.c_int64, _p, _p, _p, _p, _p, _p, _p, _p]),
    "bwpm_server_stats": (_i, [_p, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p]),
    "bwpm_server_destroy": (None, [_p]),
    "bwpm_port_power": (_i, [_i, _sz, _sz, _d, _d, _d, _d, _d, _i, _p, ctypes.POINTER(_d)]),
    "bwpm_plane_power": (_i, [_i, _sz, _sz, _d, _d, _d, _d, _p, ctypes.POINTER(_d)]),
    "bwpm_axial_focus": (_i, [_i, _sz, _sz, _d, _d, _d, _d, _p, _sz, _d, _p, ctypes.POINTER(_d),
                              ctypes.POINTER(_d), _p]),
    "bwpm_flush_l2": (_i, [_i, _sz]),
    "bwpm_step2d_noalloc": (_i, [_i, _sz, _d, _d, _d, _p, _sz, _p, _p, _d, _d, _p, _p, _p, _p]),
    "bwpm_host_register": (_i, [_p, _sz]),
    "bwpm_host_unregister": (_i, [_p]),
}


def _bind() -> None:
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args


_bind()


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    lib.bwpm_last_error(buf, 4096)
    return buf.value.decode("utf-8", "replace")


def check(status: int) -> None:
    """Raises the reference's exception type for a failed call (ValueError / RuntimeError)."""
    if status == BWPM_OK:
        return
    msg = last_error()
    if status == BWPM_EINVAL:
        raise ValueError(msg)
    raise RuntimeError(msg)


def ptr(a: np.ndarray | None) -> int | None:
    """Address of a C-contiguous array (None for None)."""
    if a is None:
        return None
    assert a.flags.c_contiguous
    return a.ctypes.data
