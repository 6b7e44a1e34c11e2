"""The C ABI library loads, exports every symbol include/ghex_b200.h declares, and reports errors
through status codes (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from ghex_b200 import _capi

HEADER = Path(__file__).resolve().parents[1] / "include" / "ghex_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^int (ghexb_\w+)\(", text, flags=re.M)))


def test_header_declares_functions():
    names = declared_functions()
    assert len(names) >= 30
    assert "ghexb_co_exchange" in names and "ghexb_handle_wait" in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    assert hasattr(_capi.lib, name), f"{name} is declared but not exported"
    assert name in _capi.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_errors():
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    _capi.call("ghexb_version", C.byref(a), C.byref(b), C.byref(c))
    assert (a.value, b.value) == (0, 1)
    rc = _capi.lib.ghexb_version(None, None, None)
    assert rc == _capi.ERR_INVALID
    assert "null" in _capi.last_error()


def test_context_without_device_and_bad_pattern():
    h = C.c_void_p()
    _capi.call("ghexb_context_create", 0, C.byref(h))
    try:
        p = C.c_void_p()
        # empty domain
        rc = _capi.lib.ghexb_pattern_create_regular(
            h, 1, _capi.int_array([0]), _capi.int_array([9]), _capi.int_array([1, 1]), _capi.int_array([1]), 1,
            _capi.int64_array([0]), _capi.int_array([5]), _capi.int_array([4]), C.byref(p))
        assert rc == _capi.ERR_INVALID
        assert "empty" in _capi.last_error()
        # repeated ids
        rc = _capi.lib.ghexb_pattern_create_regular(
            h, 1, _capi.int_array([0]), _capi.int_array([9]), _capi.int_array([1, 1]), _capi.int_array([1]), 2,
            _capi.int64_array([3, 3]), _capi.int_array([0, 5]), _capi.int_array([4, 9]), C.byref(p))
        assert rc == _capi.ERR_INVALID
        assert "repeated" in _capi.last_error()
    finally:
        _capi.lib.ghexb_context_destroy(h)


def test_field_wrap_checks():
    from ghex_b200.structured import regular as R
    ctx = R.make_context(device=0)
    hg = R.HaloGenerator(((0,), (9,)), (1,), (True,))
    p = R.make_pattern(ctx, hg, [R.DomainDescriptor(0, ((0,), (4,))), R.DomainDescriptor(1, ((5,), (9,)))])
    f = C.c_void_p()
    # unknown domain id
    rc = _capi.lib.ghexb_field_wrap(p._h, 7, _capi.F64, C.c_void_p(4096), 1, _capi.int_array([1]),
                                    _capi.int_array([7]), None, None, 1, 0, C.byref(f))
    assert rc == _capi.ERR_INCOMPATIBLE
    assert "incompatible" in _capi.last_error()
    # misaligned pointer
    rc = _capi.lib.ghexb_field_wrap(p._h, 0, _capi.F64, C.c_void_p(4100), 1, _capi.int_array([1]),
                                    _capi.int_array([7]), None, None, 1, 0, C.byref(f))
    assert rc == _capi.ERR_INVALID
    # components on a field without a component dimension
    rc = _capi.lib.ghexb_field_wrap(p._h, 0, _capi.F64, C.c_void_p(4096), 1, _capi.int_array([1]),
                                    _capi.int_array([7]), None, None, 3, 0, C.byref(f))
    assert rc == _capi.ERR_INVALID
    assert "components" in _capi.last_error()
    # a valid wrap needs no device
    _capi.call("ghexb_field_wrap", p._h, 0, _capi.F64, C.c_void_p(4096), 1, _capi.int_array([1]),
               _capi.int_array([7]), None, None, 1, 0, C.byref(f))
    _capi.lib.ghexb_field_destroy(f)


def test_ghex_module_names():
    """The module layout of GHEX's Python package: ghex.context.make_context, ghex.util.Architecture,
    and make_communication_object / make_pattern / make_field_descriptor in each grid module."""
    from ghex_b200 import unstructured
    from ghex_b200.context import context, make_context
    from ghex_b200.structured import cubed_sphere, regular
    from ghex_b200.util import Architecture
    ctx = make_context(None, False, device=0)
    assert isinstance(ctx, context) and ctx.rank() == 0 and ctx.size() == 1
    assert {a.name for a in Architecture} == {"CPU", "GPU"}
    for mod in (regular, cubed_sphere, unstructured):
        for name in ("make_communication_object", "make_pattern", "make_field_descriptor", "wrap_field",
                     "make_bulk_communication_object", "make_exchange_plan"):
            assert callable(getattr(mod, name)), (mod.__name__, name)
    assert callable(regular.make_staged_pattern) and callable(unstructured.make_communication_object_ipr)


def test_sharded_and_ipc_argument_checks():
    """Sharded plans and IPC mappings refuse bad arguments before any device call."""
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_plan_check import regular_handles
    from ghex_b200 import workloads as W
    ctx, keep, handles = regular_handles(W.config0())
    arr = (C.c_void_p * len(handles))(*handles)
    n = C.c_int64()
    local = bytes([1] * len(handles))
    # mode outside 1 (pull) and 2 (push)
    assert _capi.lib.ghexb_plan_check_sharded(ctx._h, arr, len(handles), local, 3, C.byref(n)) == _capi.ERR_INVALID
    assert "pull" in _capi.last_error()
    # locality flags are required
    assert _capi.lib.ghexb_plan_check_sharded(ctx._h, arr, len(handles), None, 1, C.byref(n)) == _capi.ERR_INVALID
    # every field local: the pull and push parts are the whole exchange
    _capi.call("ghexb_plan_check_sharded", ctx._h, arr, len(handles), local, 1, C.byref(n))
    pull = n.value
    _capi.call("ghexb_plan_check_sharded", ctx._h, arr, len(handles), local, 2, C.byref(n))
    assert n.value == pull == 52288  # the written halo cells of the 64^3, 2x2x2, halo-1 workload
    # no field local: an empty part
    _capi.call("ghexb_plan_check_sharded", ctx._h, arr, len(handles), bytes(len(handles)), 1, C.byref(n))
    assert n.value == 0
    # a handle never opened here
    assert _capi.lib.ghexb_ipc_close(bytes(_capi.IPC_HANDLE_BYTES)) == _capi.ERR_INVALID
    assert "not open" in _capi.last_error()
    p = C.c_void_p()
    assert _capi.lib.ghexb_ipc_open(bytes(_capi.IPC_HANDLE_BYTES), -1, C.byref(p)) == _capi.ERR_INVALID


def test_adjoint_tuning_range():
    assert _capi.lib.ghexb_plan_set_adjoint_tuning(None, 0) == _capi.ERR_INVALID


def test_stencil_argument_checks():
    """ghexb_stencil7 refuses bad arguments before any device call (fake addresses, never read)."""
    P = C.c_void_p * 1
    I64 = C.c_int64 * 3

    def call(dtype=_capi.F64, n=1, src=1 << 40, dst=(1 << 40) + (1 << 30), ext=(8, 8, 8), st=(1, 8, 64), halo=1):
        return _capi.lib.ghexb_stencil7(dtype, n, P(src), P(dst), I64(*ext), I64(*st), halo, 0.1, 0, None)

    assert call(n=0) == 0                                   # nothing to do, no device needed
    cases = [
        (dict(dtype=99), "float32 or float64"),
        (dict(n=-1), "negative"),
        (dict(halo=0), "halo"),
        (dict(src=0), "null"),
        (dict(src=(1 << 40) + 4), "aligned"),               # float64 data at a 4-byte boundary
        (dict(ext=(2, 8, 8)), "twice the halo"),
        (dict(ext=(8, 8, 4), halo=2), "twice the halo"),
        (dict(st=(1, 0, 64)), "positive"),
        (dict(dst=(1 << 40) + 8 * 100), "overlap"),         # inside the 512-element input
    ]
    for kw, msg in cases:
        assert call(**kw) == _capi.ERR_INVALID, kw
        assert msg in _capi.last_error(), (kw, _capi.last_error())
