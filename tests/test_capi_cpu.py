"""CPU-side checks of the C ABI: the library builds, loads and exports every
function include/sincgpu.h declares; argument validation fails cleanly without
touching a GPU."""
import ctypes as C

import pytest


def test_library_exports_every_declared_symbol(built_lib):
    import sincgpu
    lib = sincgpu.load_library()
    declared = sincgpu.exported_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert missing == []


def test_bindings_cover_header(built_lib):
    from sincgpu import capi
    assert sorted(capi._SIGS) == sorted(capi.exported_symbols())


def test_null_context_is_an_error_not_a_crash(built_lib):
    import sincgpu
    lib = sincgpu.load_library()
    rc = lib.sincgpu_mult_ke(None, None, None, 1)
    assert rc == 1  # SINCGPU_EINVAL
    assert b"null context" in lib.sincgpu_last_error()


def test_create_rejects_bad_sizes_before_any_device_work(built_lib):
    import sincgpu
    lib = sincgpu.load_library()
    h = C.c_void_p()
    cs = (C.c_int * 3)(0, 0, 0)
    z = (C.c_double * 1)(1.0)
    assert lib.sincgpu_create(C.byref(h), 41, 0.25, 17, cs, z, 10, 240, 40, 0, 0) == 6  # numcenters
    assert lib.sincgpu_create(C.byref(h), 41, 0.25, 1, cs, z, 10, 240, 0, 0, 0) == 1   # toothnsmall
    assert not h


def test_missing_library_fails_loudly(tmp_path):
    from sincgpu import capi
    with pytest.raises(ImportError, match="no CPU fallback"):
        capi.load_library(tmp_path / "libsincgpu.so")
