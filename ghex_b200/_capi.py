"""ctypes binding of libghex_b200.so (the C ABI declared in include/ghex_b200.h).

The library is loaded from the package directory. There is no fallback: importing this module
raises ImportError when the library has not been built (python -m ghex_b200.build).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libghex_b200.so"

if not LIB_PATH.exists():
    raise ImportError(
        f"{LIB_PATH} is missing: build the CUDA extension with `python -m ghex_b200.build`"
    )

lib = C.CDLL(str(LIB_PATH))


def _make_release(library):
    def release(name: str, handle) -> None:
        """Destroys a handle with ghexb_<...>_destroy; the library is held by this closure, so the
        call also works while the interpreter tears modules down."""
        if handle:
            try:
                getattr(library, name)(handle)
            except Exception:
                pass
    return release


release = _make_release(lib)

OK = 0
ERR_INVALID = 1
ERR_CUDA = 2
ERR_BUSY = 3
ERR_INCOMPATIBLE = 4
ERR_RANGE = 5
ERR_ALLOC = 6
ERR_INTERNAL = 7

F32, F64, I32, I64, U8, U16 = 0, 1, 2, 3, 4, 5
FORM_BATCHED, FORM_PER_FIELD, FORM_PER_BOX = 0, 1, 2
IPC_HANDLE_BYTES = 64  # GHEXB_IPC_HANDLE_BYTES

_vp = C.c_void_p
_i = C.c_int
_i64 = C.c_int64
_pi = C.POINTER(C.c_int)
_pi64 = C.POINTER(C.c_int64)


class PlanInfo(C.Structure):
    _fields_ = [
        ("num_fields", C.c_int64),
        ("num_descriptors", C.c_int64),
        ("num_tiles", C.c_int64),
        ("halo_elements", C.c_int64),
        ("algorithmic_bytes", C.c_int64),
        ("index_bytes", C.c_int64),
        ("adjoint_launches", C.c_int64),
        ("adjoint_cells", C.c_int64),
        ("elems_per_thread", C.c_int32),
        ("block", C.c_int32),
        ("grid", C.c_int32),
        ("pairs", C.c_int32),
        ("use_pairs", C.c_int32),
        ("staged_mode", C.c_int32),
        ("staged_boxes", C.c_int32),
        ("staged_items", C.c_int32),
        ("staged_maps", C.c_int32),
        ("stages", C.c_int32),
        ("stage_bytes", C.c_int32),
        ("stage_consumers", C.c_int32),
        ("stage_ctas_per_sm", C.c_int32),
        ("gather_scale", C.c_int32),
        ("bulk_share", C.c_int32),
        ("bulk_tiles", C.c_int32),
        ("gather_bulk", C.c_int32),
        ("gather_bulk_tiles", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# name -> argtypes; every function returns int status
SIGNATURES = {
    "ghexb_last_error": [C.c_char_p, C.c_size_t],
    "ghexb_version": [_pi, _pi, _pi],
    "ghexb_context_create": [_i, C.POINTER(_vp)],
    "ghexb_context_destroy": [_vp],
    "ghexb_pattern_create_regular": [_vp, _i, _pi, _pi, _pi, _pi, _i, _pi64, _pi, _pi, C.POINTER(_vp)],
    "ghexb_pattern_create_regular_staged": [_vp, _i, _pi, _pi, _pi, _pi, _i, _pi64, _pi, _pi, _pi64, C.POINTER(_vp)],
    "ghexb_pattern_create_cubed_sphere": [_vp, _i, _i, _pi, _i, _pi, _pi, _pi, _pi, _pi, C.POINTER(_vp)],
    "ghexb_pattern_create_unstructured": [_vp, _i, _pi64, _pi64, _pi64, _pi64, _pi64, _pi64, _pi64,
                                          C.POINTER(_vp)],
    "ghexb_pattern_create_unstructured_hinted": [_vp, _i, _pi64, _pi64, _pi64, _pi64, _pi64, _pi64, _pi64, _pi64,
                                                 _pi64, _pi64, C.POINTER(_vp)],
    "ghexb_pattern_destroy": [_vp],
    "ghexb_pattern_num_domains": [_vp, _pi],
    "ghexb_pattern_domain_id": [_vp, _i, _pi64],
    "ghexb_pattern_max_tag": [_vp, _pi],
    "ghexb_pattern_num_spaces": [_vp, _i, _i, _pi],
    "ghexb_pattern_space": [_vp, _i, _i, _i, _pi, _pi, _pi, _pi, _pi],
    "ghexb_pattern_space_indices": [_vp, _i, _i, _i, _pi, _pi64, _i64, _pi64],
    "ghexb_field_wrap": [_vp, _i64, _i, _vp, _i, _pi, _pi, _pi, _pi64, _i, _i, C.POINTER(_vp)],
    "ghexb_field_wrap_unstructured": [_vp, _i64, _i, _vp, _i64, _i, _i64, C.POINTER(_vp)],
    "ghexb_field_destroy": [_vp],
    "ghexb_host_register": [_vp, C.c_size_t, _pi],
    "ghexb_host_unregister": [_vp],
    "ghexb_co_create": [_vp, C.POINTER(_vp)],
    "ghexb_co_create_ipr": [_vp, C.POINTER(_vp)],
    "ghexb_co_destroy": [_vp],
    "ghexb_co_exchange": [_vp, C.POINTER(_vp), _i, _vp, C.POINTER(_vp)],
    "ghexb_handle_wait": [_vp],
    "ghexb_handle_is_ready": [_vp, _pi],
    "ghexb_handle_destroy": [_vp],
    "ghexb_plan_create": [_vp, C.POINTER(_vp), _i, C.POINTER(_vp)],
    "ghexb_plan_create_ipr": [_vp, C.POINTER(_vp), _i, C.POINTER(_vp)],
    "ghexb_plan_destroy": [_vp],
    "ghexb_plan_check": [_vp, C.POINTER(_vp), _i, _pi64],
    "ghexb_plan_get_info": [_vp, C.POINTER(PlanInfo)],
    "ghexb_plan_set_staged": [_vp, _i, _i, _i, _i, _i],
    "ghexb_host_alloc": [C.c_size_t, C.POINTER(_vp)],
    "ghexb_host_is_mapped": [_vp, C.c_size_t, _pi],
    "ghexb_host_free": [_vp],
    "ghexb_calibrate_rows": [_vp, _vp, C.c_int64, _i, C.c_int64, C.c_int64, _i, _i, _vp],
    "ghexb_plan_staged_status": [_vp, C.POINTER(C.c_uint)],
    "ghexb_plan_set_adjoint_tuning": [_vp, _i],
    "ghexb_plan_set_bulk": [_vp, _i],
    "ghexb_plan_set_adjoint_bulk": [_vp, _i],
    "ghexb_plan_create_sharded": [_vp, C.POINTER(_vp), _i, C.c_char_p, _i, C.POINTER(_vp)],
    "ghexb_plan_check_sharded": [_vp, C.POINTER(_vp), _i, C.c_char_p, _i, _pi64],
    "ghexb_ipc_export": [_vp, C.c_char_p, _pi64],
    "ghexb_ipc_open": [C.c_char_p, _i64, C.POINTER(_vp)],
    "ghexb_ipc_close": [C.c_char_p],
    "ghexb_plan_dram_floor": [_vp, C.POINTER(_vp), _i, _i, C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "ghexb_plan_set_tuning": [_vp, _i, _i, _i],
    "ghexb_plan_launch": [_vp, _i, _vp],
    "ghexb_plan_graph_launch": [_vp, _vp],
    "ghexb_plan_adjoint_launch": [_vp, _vp],
    "ghexb_plan_autotune": [_vp, _vp, _i, C.POINTER(PlanInfo)],
    "ghexb_exchange_noalloc": [_vp, C.POINTER(_vp), _i, _vp],
    "ghexb_plan_rebind": [_vp, C.POINTER(_vp), _i, _vp],
    "ghexb_stencil7": [_i, _i, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(C.c_int64), C.POINTER(C.c_int64), _i,
                       C.c_double, _i, _vp],
}

for _name, _args in SIGNATURES.items():
    _fn = getattr(lib, _name)
    _fn.argtypes = _args
    _fn.restype = C.c_int


class GhexError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib.ghexb_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != OK:
        raise GhexError(rc, last_error())


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args))


def int_array(values) -> C.Array:
    values = [int(v) for v in values]
    return (C.c_int * max(1, len(values)))(*values)


def int64_array(values):
    """An int64 buffer for a C call: numpy arrays are passed without copying element by element
    (the returned object keeps the memory alive for the duration of the call)."""
    try:
        import numpy as np
        if isinstance(values, np.ndarray) or (isinstance(values, (list, tuple)) and len(values) > 4096):
            arr = np.ascontiguousarray(np.asarray(values, dtype=np.int64))
            if arr.size == 0:
                arr = np.zeros(1, dtype=np.int64)
            return _NumpyArg(arr, C.c_int64)
    except ImportError:  # pragma: no cover
        pass
    values = [int(v) for v in values]
    return (C.c_int64 * max(1, len(values)))(*values)


class _NumpyArg:
    """Wraps a numpy array as a ctypes pointer argument (ctypes calls `_as_parameter_`)."""

    def __init__(self, arr, ctype):
        self._arr = arr
        self._as_parameter_ = arr.ctypes.data_as(C.POINTER(ctype))
