"""CPU tests of the C ABI: the libraries load, every declared entry point is
exported, the ctypes mirrors match the C layouts, and argument validation
reports errors without touching a GPU."""
import ctypes as ct
import os
import re
import subprocess

import pytest

import dhara_b200 as db
from dhara_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dhara_[a-z0-9_]+)\s*\(", text)))


def exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_library_exports_every_declared_symbol():
    syms = exported(db.LIB_PATH)
    missing = [s for s in declared("dhara_gpu.h") if s not in syms]
    assert not missing, missing
    assert not any("internal" in s for s in syms)


def test_dropin_library_exports():
    path = os.path.join(ROOT, "dhara_b200", "libdhara_b200.so")
    syms = exported(path)
    for s in ("_Z19SubsurfaceFlowModel", "_Z17OverlandFlowModel"):
        assert any(x.startswith(s) for x in syms), s


def test_abi_version_and_layouts():
    L = db.lib()
    assert L.dhara_abi_version() == 1
    p = db.default_params(4, 5, 6, 1.0, 1.0, 0.05, 60.0)
    assert p.struct_size == ct.sizeof(db.Params)
    assert ct.sizeof(db.Diagnostics) == 200


def test_default_params_match_python_mirror():
    c = db.default_params(7, 8, 9, 1.2, 1.2, 0.2, 1800.0)
    py = _abi.make_params(7, 8, 9, dx=1.2, dy=1.2, dz=0.2, dt=1800.0)
    for name, _ in db.Params._fields_:
        if name.startswith("reserved"):
            continue
        assert getattr(c, name) == getattr(py, name), name


@pytest.mark.parametrize("mutate,code,text", [
    (lambda p: setattr(p, "struct_size", 8), 1, "struct_size"),
    (lambda p: setattr(p, "nz", 100), 4, "nz=100"),
    (lambda p: setattr(p, "dt", -1.0), 1, "dt"),
    (lambda p: setattr(p, "n", 0.9), 1, "van Genuchten"),
    (lambda p: setattr(p, "am", 1.5), 1, "am"),
    (lambda p: setattr(p, "precision", 7), 1, "precision"),
])
def test_create_validates_before_touching_the_gpu(mutate, code, text):
    p = _abi.make_params(8, 8, 8)
    mutate(p)
    h = ct.c_void_p()
    rc = db.lib().dhara_create(ct.byref(p), 1, 0, ct.byref(h))
    assert rc == code
    assert text in db.lib().dhara_last_error().decode()


def test_mixed_precisions_in_one_handle_rejected():
    a = _abi.make_params(8, 8, 8, precision=_abi.FP64)
    b = _abi.make_params(8, 8, 8, precision=_abi.MIXED)
    arr = (db.Params * 2)(a, b)
    h = ct.c_void_p()
    assert db.lib().dhara_create(arr, 2, 0, ct.byref(h)) == 1


def test_null_arguments():
    L = db.lib()
    assert L.dhara_create(None, 1, 0, None) == 1
    assert L.dhara_step(None, 1, 0) == 1
    assert L.dhara_destroy(None) == 0
    n = ct.c_int64(-1)
    assert L.dhara_checkpoint_size(None, ct.byref(n)) == 1
    assert L.dhara_checkpoint(None, None, 0) == 1
    assert L.dhara_restore(None, None, 0) == 1


def test_bounded_wait_selftest_validates_before_touching_the_gpu():
    """The self-check's limit is validated on the host: out-of-range limits
    and a NULL result pointer are rejected without a device."""
    L = db.lib()
    out = ct.c_int(7)
    for bad in (0.0, -1.0, 1e9, float("nan")):
        assert L.dhara_selftest_bounded_wait(0, bad, ct.byref(out)) == 1
        assert b"limit_ms" in L.dhara_last_error()
    assert L.dhara_selftest_bounded_wait(0, 100.0, None) == 1


def test_oracle_library_loads():
    import oracle
    L = oracle.lib()
    assert L.oracle_get_threads() >= 1
