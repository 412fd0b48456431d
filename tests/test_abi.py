"""The C-ABI library loads and exports every entry point that
include/koral_b200.h declares (no GPU needed: nothing is called)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "koral_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(kgpu_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "kgpu_op_explicit" in syms and "kgpu_calc_u2p" in syms and len(syms) > 20


def test_library_exports_every_declared_symbol(kgpu):
    lib = ctypes.CDLL(kgpu.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version(kgpu):
    assert kgpu.lib().kgpu_abi_version() == 1


def test_invalid_config_rejected_without_gpu(kgpu):
    # argument checks run before any CUDA call
    cfg = kgpu.default_config(16, 16, 1)
    cfg.nv = 7
    h = ctypes.c_void_p()
    assert kgpu.lib().kgpu_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
    cfg = kgpu.default_config(16, 16, 1, int_order=3)
    assert kgpu.lib().kgpu_create(ctypes.byref(cfg), ctypes.byref(h)) == -1
