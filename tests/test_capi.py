"""The C-ABI library loads and exports every entry point include/*.h declares.
CPU only: no compute call is made here."""
import ctypes as C
import os
import re

import pytest

import slsimlib_b200 as glb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(inc, f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(glb_[A-Za-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    L = glb.load_library()
    decl = declared_symbols()
    assert decl, "no declarations found"
    missing = [s for s in sorted(decl) if not hasattr(L, s)]
    assert not missing, missing
    assert set(glb.EXPORTED) == decl


def test_version_and_error_strings():
    L = glb.load_library()
    assert b"sm_100a" in L.glb_version()
    assert L.glb_set_option(12345, 1) == glb.GLB_ERR_ARG
    assert b"unknown option" in L.glb_last_error()


def _has_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_device(), reason="checks the no-device error path")
def test_no_cpu_fallback_without_device():
    with pytest.raises(glb.GlamerError) as e:
        glb.Lens(2.0)
    assert e.value.code == glb.GLB_ERR_NO_DEVICE


def test_argument_errors_before_any_device_work():
    L = glb.load_library()
    out = C.c_void_p()
    # non-flat cosmology is refused (MultiPlane/lens.cpp:63-67)
    assert L.glb_lens_create(2.0, 0.3, 0.6, 0.7, C.byref(out)) == glb.GLB_ERR_ARG
    assert L.glb_halo_nsie(1e13, 0.5, 250.0, 0.0, 1.5, 0.0, C.byref(out)) == glb.GLB_ERR_ARG
    assert L.glb_halo_nfw(1e14, 1.0, 0.3, 5.0, 0.5, 0.0, C.byref(out)) == glb.GLB_ERR_UNSUPPORTED
