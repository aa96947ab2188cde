"""CPU tests of the C-ABI library: it loads, exports exactly the entry points
include/reyn_b200.h declares, and rejects invalid arguments with status codes
before touching a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

import reyn_b200 as rb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "reyn_b200.h")


def header_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(reyn_[a-z0-9_]+)\s*\(", src)))


def test_library_loads():
    L = rb.lib()
    assert L.reyn_abi_version() == 1


def test_exports_every_declared_symbol():
    declared = header_symbols()
    assert len(declared) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", rb.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted(set(re.findall(r" T (reyn_[a-z0-9_]+)", out)))
    assert exported == declared
    assert sorted(rb.declared_symbols()) == declared


def test_invalid_arguments_return_status():
    L = rb.lib()
    h = ctypes.c_void_p()
    f3 = rb._f3
    assert L.reyn_grid_create(f3([0, 0, 0]), f3([1, 1, 1]), -1.0, 0.5, 0, ctypes.byref(h)) == \
        rb.ERR_INVALID
    assert b"radius" in L.reyn_last_error()
    assert L.reyn_grid_create(f3([0, 0, 0]), f3([1, 1, 1]), 0.1, 0.7, 0, ctypes.byref(h)) == \
        rb.ERR_INVALID
    assert L.reyn_grid_create(f3([0, 0, 0]), f3([-1, 1, 1]), 0.1, 0.5, 0, ctypes.byref(h)) == \
        rb.ERR_INVALID
    assert L.reyn_grid_create(f3([0, 0, float("nan")]), f3([1, 1, 1]), 0.1, 0.5, 0,
                              ctypes.byref(h)) == rb.ERR_INVALID
    assert L.reyn_grid_create(f3([0, 0, 0]), f3([1, 1, 1]), 0.1, 0.5, 7, ctypes.byref(h)) == \
        rb.ERR_INVALID
    p = rb.Params()
    assert L.reyn_params_reference(2, 9, 0.01, 1000.0, 0.01, ctypes.byref(p)) == rb.ERR_INVALID
    assert L.reyn_params_reference(5, 0, 0.01, 1000.0, 0.01, ctypes.byref(p)) == rb.ERR_INVALID
    assert L.reyn_params_reference(2, 0, 0.01, 1000.0, 0.01, ctypes.byref(p)) == rb.OK
    assert (p.eta, p.min_iter, p.omega, p.warmstart) == (pytest.approx(0.005), 3, 0.5, 1)
    assert tuple(p.g) == (0.0, pytest.approx(-9.81), 0.0)
    bad = rb.Params.from_buffer_copy(p)
    bad.omega = 2.5
    assert L.reyn_solver_create(2, ctypes.byref(bad), 10, ctypes.byref(h)) == rb.ERR_INVALID
    bad = rb.Params.from_buffer_copy(p)
    bad.h = 0.0
    assert L.reyn_solver_create(2, ctypes.byref(bad), 10, ctypes.byref(h)) == rb.ERR_INVALID
    assert L.reyn_particles_create(10, -1.0, ctypes.byref(h)) == rb.ERR_INVALID
    assert L.reyn_kernel_eval(7, 1.0, None, None, None, 0, None, None, None, None, None) == \
        rb.ERR_INVALID
    assert L.reyn_solver_step(None, None, None, None, 1e-3, None, None) == rb.ERR_INVALID
    assert L.reyn_enforce_bounds(None, f3([0, 0, 0]), f3([1, 1, 1]), None) == rb.ERR_INVALID


def test_reference_params_per_scheme():
    p = rb.reference_params(rb.PCISPH, rb.B3, 0.01, 1000.0, 0.01)
    assert p.eta == pytest.approx(0.001) and p.min_iter == 3
    p = rb.reference_params(rb.SESPH, rb.B3, 0.01, 1000.0, 0.01)
    assert p.k_sesph == 500.0


def test_header_is_plain_c_and_adapter_compiles(tmp_path):
    """include/reyn_b200.h compiles as strict C99 (the ABI a cgo/ctypes/JNI
    binding sees), and the C++ adapter include/reyn_b200.hpp as C++17."""
    c = tmp_path / "abi.c"
    c.write_text('#include "reyn_b200.h"\nint main(void) { return reyn_abi_version() != 1; }\n')
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    "-I" + os.path.join(ROOT, "include"), "-c", str(c), "-o",
                    str(tmp_path / "abi.o")], check=True)
    cc = tmp_path / "adapter.cpp"
    cc.write_text('#include "reyn_b200.hpp"\nint main() { return 0; }\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror",
                    "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
                    "-fsyntax-only", str(cc)], check=True)
