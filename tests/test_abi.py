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


def build_rk2_loop(kgpu, out_dir):
    """Compiles tests/abi/rk2_loop.c (KORAL's RK2 loop written against the
    header) with gcc and links it to the library."""
    import subprocess
    exe = os.path.join(str(out_dir), "rk2_loop")
    libdir = os.path.dirname(kgpu.LIB_PATH)
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "abi", "rk2_loop.c"), "-L", libdir, "-lkoral_b200",
                           "-Wl,-rpath," + libdir, "-o", exe])
    return exe


def test_rk2_loop_program_compiles_and_links(kgpu, tmp_path):
    """The host-side loop compiles as C99 against include/koral_b200.h and
    links against every symbol it names."""
    assert os.path.exists(build_rk2_loop(kgpu, tmp_path))


def test_struct_layouts_match_python_mirrors(kgpu, tmp_path):
    """The ctypes structures of koral_b200/__init__.py have the sizes and
    field offsets a C compiler gives the header's structs (gcc on
    tests/abi/layout.c)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    exe = str(tmp_path / "layout")
    subprocess.check_call([cc, "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "abi", "layout.c"),
                           "-o", exe])
    c = dict(line.rsplit(" ", 1) for line in subprocess.check_output([exe], text=True).splitlines())
    c = {k: int(v) for k, v in c.items()}
    py = {"kgpu_config": kgpu.Config, "kgpu_torus_params": kgpu.TorusParams, "kgpu_rad_params": kgpu.RadParams,
          "kgpu_rad_solver_opts": kgpu.SolverOpts, "kgpu_tuning": kgpu.Tuning,
          "kgpu_scalars_params": kgpu.ScalarsParams}
    for name, cls in py.items():
        assert ctypes.sizeof(cls) == c[name], name
    for key, off in c.items():
        if "." not in key:
            continue
        name, field = key.split(".")
        assert getattr(py[name], field).offset == off, key
