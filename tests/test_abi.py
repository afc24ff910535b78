"""CPU checks of the C ABI boundary: the library builds for sm_100a, loads,
and exports every function include/femh.h declares; host-side argument
checks fail cleanly without a GPU."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "femh.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(femh_[a-zA-Z_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from fem_b200 import build
    path = build.build()
    return ctypes.CDLL(path)


def test_header_declares_expected_api():
    names = _declared()
    for n in ("femh_create", "femh_homogenize", "femh_homogenize_grad", "femh_homogenize_batch",
              "femh_dCdrho", "femh_full_field", "femh_apply_operator", "femh_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    for name in _declared():
        assert hasattr(lib, name), name


def test_python_binding_lists_all_exports():
    import fem_b200
    assert sorted(fem_b200.EXPORTS) == _declared()


def test_config_default_matches_binding(lib):
    import dataclasses
    import fem_b200
    from fem_b200.femh import _Config
    c = _Config()
    assert lib.femh_config_default(ctypes.byref(c)) == 0
    d = fem_b200.Config()
    for f in dataclasses.fields(d):
        assert getattr(c, f.name) == pytest.approx(getattr(d, f.name)), f.name


def test_bad_config_rejected_before_device_use(lib):
    from fem_b200.femh import _Config
    lib.femh_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(_Config)]
    for field, value in (("nu", 0.7), ("cheb_ratio", 0.5), ("cheb_ratio", -2.0), ("stencil_variant", 8)):
        c = _Config()
        lib.femh_config_default(ctypes.byref(c))
        setattr(c, field, value)
        h = ctypes.c_void_p()
        assert lib.femh_create(ctypes.byref(h), ctypes.byref(c)) == 1, field   # FEMH_E_ARG
        assert not h.value


def test_null_handle_is_an_argument_error(lib):
    lib.femh_homogenize.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3 + [
        ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    assert lib.femh_homogenize(None, 4, 4, 4, 0.25, None, 0, None, None) == 1
    lib.femh_kernel_launches.restype = ctypes.c_longlong
    assert lib.femh_kernel_launches(None) == -1
