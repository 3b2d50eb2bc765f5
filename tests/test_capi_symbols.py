"""The C-ABI library loads without a GPU and exports every entry point that
include/dvg.h declares; without a device, context creation fails loudly."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "diffvg-rs_b200")
LIB = os.path.join(PKG, "libdvg_b200.so")


def _declared(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dvg_[a-z0-9_]+)\s*\(", text)))


def _ensure_built():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", PKG], check=True)


def test_header_declares_entry_points():
    names = _declared(os.path.join(ROOT, "include", "dvg.h"))
    for n in ("dvg_context_create", "dvg_scene_upload", "dvg_render", "dvg_render_backward",
              "dvg_render_device", "dvg_render_backward_device", "dvg_fwd_bwd_l2_device"):
        assert n in names


def test_library_exports_every_declared_symbol():
    _ensure_built()
    lib = C.CDLL(LIB)
    for header in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not header.endswith(".h"):
            continue
        for name in _declared(os.path.join(ROOT, "include", header)):
            assert hasattr(lib, name), f"{name} declared in include/{header} but not exported"


def test_abi_version_and_no_device_error():
    _ensure_built()
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present; the no-device path is not reachable")
    lib = C.CDLL(LIB)
    lib.dvg_abi_version.restype = C.c_uint32
    assert lib.dvg_abi_version() == 2
    ctx = C.c_void_p()
    lib.dvg_context_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
    st = lib.dvg_context_create(0, C.byref(ctx))
    assert st == 6  # DVG_ERR_NO_DEVICE: no silent CPU fallback
    lib.dvg_last_error.restype = C.c_char_p
    assert b"no CUDA device" in lib.dvg_last_error()
