"""The C-ABI boundary: the engine library loads without a GPU and exports every
function include/*.h declares; the ctypes mirror declares the same set."""
import ctypes
import os
import re

from cppqed_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("cqg.h", "cqg_model.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(cqg_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(engine):
    lib = ctypes.CDLL(engine.engine.LIB_PATH)
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_mirror_covers_the_headers():
    assert declared_functions() == set(A.ENGINE_PROTOTYPES)


def test_abi_version_and_error_channel(engine):
    lib = engine.lib()
    assert lib.cqg_abi_version() == 5
    h = ctypes.c_void_p()
    rc = lib.cqg_model_create(b"NoSuchScript", 0, None, ctypes.byref(h))
    assert rc == A.CQG_E_INVALID
    assert b"unknown script" in lib.cqg_last_error()


def test_device_entry_points_fail_cleanly_without_device(engine):
    if engine.device_count() > 0:
        return
    m = engine.Model("PTLA_C++QED", [])
    try:
        engine.System(m.desc)
    except engine.EngineError as e:
        assert e.code == A.CQG_E_NODEVICE
    else:
        raise AssertionError("system creation must fail without a device")
