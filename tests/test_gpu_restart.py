"""Restart files in the reference's serial format (fileop.c:910-1111).

The GPU writes the state the reference holds; the files must equal the
reference's own, byte for byte.  The GPU reads the reference's file; the
domain's primitives and the conserved variables recomputed from them must
equal what the reference's own reader leaves.  Both the magnetised torus
(9 variables) and the radiative torus (13) are checked.
"""
import ctypes
import os
import shutil

import numpy as np
import pytest

from conftest import ref_lib_available

pytestmark = pytest.mark.gpu

CASES = [("libkref_fmtorus_small.so", 9), ("libkref_radtorus_small.so", 13)]


def make_gpu(kgpu, R, nv):
    ph = R.physics()
    cfg = kgpu.default_config(R.nx, R.ny, R.nz, ng=R.ng, nv=nv, int_order=kgpu.MP5, fluxmethod=kgpu.HLL,
                              axisym_metric=int(ph["axisym"]),
                              bc=(kgpu.BC_OUTFLOW, kgpu.BC_REFLECT, kgpu.BC_PERIODIC_COPY),
                              gamma=ph["gamma"], tsteplim=ph["tsteplim"], rhofloor=ph["rhofloor"],
                              uurhoratiomin=ph["uurhoratiomin"], uurhoratiomax=ph["uurhoratiomax"],
                              b2rhoratiomax=ph["b2rhoratiomax"], gammamaxhd=ph["gammamaxhd"],
                              u2pconv=ph["u2pconv"])
    s = kgpu.Subdomain(cfg)
    s.upload_grid(*R.grid_faces())
    s.upload_metric(*R.metric_tables())
    if nv == 13:
        s.set_radiation(kgpu.rad_params(mass=1.e16, gamma=ph["gamma"]))
    return s


def reference_copy(oracle, lib, tmp_path, tag):
    dst = str(tmp_path / f"{tag}_{lib}")
    shutil.copy(os.path.join(oracle.REF_DIR, lib), dst)
    R = oracle.RefKoral(dst)
    R.init()
    return R


@pytest.mark.parametrize("lib,nv", CASES)
def test_restart_files_equal_and_read_back(kgpu, oracle, tmp_path, lib, nv):
    if not ref_lib_available(lib):
        pytest.skip(f"{lib} not built")
    R = reference_copy(oracle, lib, tmp_path, "a")
    R.step(3)
    t = 0.375   # printed exactly by the header's %10.6e
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    ours.mkdir()
    theirs.mkdir()
    # the reference's writer
    ctypes.c_int.in_dll(R.L, "nfout1").value = 7
    ctypes.c_int.in_dll(R.L, "nfout2").value = 2
    R.L.fprint_restartfile_bin.argtypes = [ctypes.c_double, ctypes.c_char_p]
    R.L.fprint_restartfile_bin(t, str(theirs).encode())
    # ours, from the same state on the device
    s = make_gpu(kgpu, R, nv)
    s.upload_state(R.array("u").copy(), R.array("p").copy())
    s.write_restart(str(ours), 7, t, nout2=2, problem=201)
    for name in ("res0007.head", "res0007.dat"):
        a = (ours / name).read_bytes()
        b = (theirs / name).read_bytes()
        assert a == b, name
    assert os.path.realpath(ours / "reslast.dat") == str(ours / "res0007.dat")
    # reading the reference's file: the reference's own reader on a second
    # instance, ours on a fresh context
    R2 = reference_copy(oracle, lib, tmp_path, "b")
    R2.L.fread_restartfile_bin.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
    tr = ctypes.c_double()
    assert R2.L.fread_restartfile_bin(7, str(theirs).encode(), ctypes.byref(tr)) == 0
    s2 = make_gpu(kgpu, R2, nv)
    s2.upload_state(R2.array("u").copy(), R2.array("p").copy())
    tg, nnext, n2 = s2.read_restart(str(theirs), 7)
    assert tg == tr.value and nnext == 8 and n2 == 2
    ug, pg = s2.download_state()
    g = R.ng
    dom = (slice(g, g + R.nz), slice(g, g + R.ny), slice(g, g + R.nx))
    assert np.array_equal(pg[dom], R2.array("p")[dom])
    assert np.array_equal(ug[dom], R2.array("u")[dom])
    # reslast
    tl, _, _ = s2.read_restart(str(ours), -1)
    assert tl == tg
