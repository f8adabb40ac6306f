"""CPU: the C-ABI library loads and exports everything include/*.h declares;
host-side argument checks fail loudly without touching a GPU."""
import ctypes as C
import os
import re

import pytest

import merbit_b200 as mb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    names = re.findall(r"\b(merbit_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = mb.lib()
    names = _declared("merbit.h")
    assert "merbit_spmv" in names and "merbit_tile_build" in names
    for n in names:
        assert hasattr(L, n), n


def test_python_binding_covers_header():
    assert set(_declared("merbit.h")) <= set(mb.SIGNATURES)


def test_measurement_header_exported_and_bound():
    L = mb.lib()
    names = _declared("merbit_bench.h")
    assert names == ["merbit_bench_gather"]
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(mb.BENCH_SIGNATURES)
    assert L.merbit_bench_gather(None, 0, None, 0, None, 0, None) == 1  # MERBIT_ERR_INVALID


def test_synth_library_exports():
    from merbit_b200 import synth

    L = synth.lib()
    for n in _declared("merbit_synth.h"):
        assert hasattr(L, n), n


def test_status_strings():
    L = mb.lib()
    for s in range(7):
        assert L.merbit_status_string(s).decode().startswith("MERBIT")


def test_host_argument_checks_without_gpu():
    L = mb.lib()
    plan = C.c_void_p()
    # null plan out-pointer
    assert L.merbit_plan_create(None, 1, 1, 0, None, None, None, 0, 0, None) == 1
    # negative sizes
    assert L.merbit_plan_create(C.byref(plan), -1, 1, 0, None, None, None, 0, 0, None) == 1
    # unknown dtype
    assert L.merbit_plan_create(C.byref(plan), 1, 1, 0, C.c_void_p(16), None, None, 9, 0,
                                None) == 1
    # nrow + nnz beyond the int32 merge path
    assert L.merbit_plan_create(C.byref(plan), 2**31 - 1, 4, 2**31 - 1, C.c_void_p(16),
                                C.c_void_p(16), C.c_void_p(16), 0, 0, None) == 3
    assert b"int32" in L.merbit_last_error_detail()
    t, l = C.c_int32(), C.c_int32()
    assert L.merbit_tile_dims(100, 1000, 14, C.byref(t), C.byref(l)) == 0
    assert (t.value, l.value) == (3, 79)
    assert L.merbit_tile_dims(100, 1000, 0, C.byref(t), C.byref(l)) == 1
    assert L.merbit_tile_dims(100, 1000, 43, C.byref(t), C.byref(l)) == 1
    assert L.merbit_spmv(None, 1.0, None, 0.0, None, None) == 1
    assert L.merbit_plan_destroy(None) == 0


def test_error_is_raised_as_exception():
    with pytest.raises(mb.MerbitError) as ei:
        mb._check(1)
    assert ei.value.status == 1
