"""The polar-axis corrections of do_correct (finite.c:605-640) against
reference builds of the small tori compiled with CORRECT_POLARAXIS,
CORRECT_POLARAXIS_3D and SMOOTH_POLARAXIS (NCCORRECTPOLAR = 2).

* do_correct alone, from the reference's state after three steps: every
  variable of every cell equals the reference's after its do_correct, bit
  for bit except the entropy of the corrected cells' conserved state (p2u
  goes through log and pow; 1e-12 relative).
* Whole time steps, each started from the reference's state: conserved
  variables and primitives within 1e-12 relative, as the torus's own
  per-step test holds them, corrected cells, their field-only inversion
  and the zeroed polar EMFs included.
* The radiative torus with CORRECT_POLARAXIS: do_correct, op_explicit and
  calc_u2p against the reference's (the M1 inversion goes through pow:
  radiation primitives within 1e-11, as in the radiative torus's own
  test), and op_implicit leaves the corrected cells untouched.
"""
import ctypes

import numpy as np
import pytest

from conftest import ref_lib_available

pytestmark = pytest.mark.gpu

CASES = [("libkref_fmtorus_polar_small.so", 1), ("libkref_fmtorus_polar3d_small.so", 2),
         ("libkref_fmtorus_smooth_small.so", 4)]
RADLIB = "libkref_radtorus_polar_small.so"


def make_pair(kgpu, oracle, lib, nv, flags):
    R = oracle.RefKoral(lib)
    R.init()
    R.step(3)
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
    c, f = R.rhofloor_table()
    s.set_density_floor(c, f)
    if nv == 13:
        s.set_radiation(kgpu.rad_params(mass=kgpu.RADTORUS_MASS, gamma=ph["gamma"]))
    s.set_polar_correction(flags, 2)
    s.upload_state(R.array("u").copy(), R.array("p").copy())
    s.tstepdenmax = R.scalar("tstepdenmax")
    R.L.op_explicit.argtypes = [ctypes.c_double, ctypes.c_double]
    R.L.op_implicit.argtypes = [ctypes.c_double, ctypes.c_double]
    return R, s


def dom(R, a):
    g = R.ng
    return a[g:g + R.nz, g:g + R.ny, g:g + R.nx, :]


def close(a, b, rtol):
    scale = np.abs(b).reshape(-1, b.shape[-1]).max(axis=0)
    return np.abs(a - b) <= rtol * (np.abs(b) + 1e-6 * scale)


@pytest.mark.parametrize("lib,flags", CASES)
def test_do_correct_matches_reference(kgpu, oracle, lib, flags):
    if not ref_lib_available(lib):
        pytest.skip(f"{lib} not built")
    R, s = make_pair(kgpu, oracle, lib, 9, flags)
    u0 = R.array("u").copy()
    R.L.do_correct()
    s.do_correct()
    u, p = s.download_state()
    ur, pr = R.array("u"), R.array("p")
    assert np.array_equal(dom(R, p), dom(R, pr))
    nonent = [0, 1, 2, 3, 4, 6, 7, 8]
    assert np.array_equal(dom(R, u)[..., nonent], dom(R, ur)[..., nonent])
    assert close(dom(R, u), dom(R, ur), 1e-12).all()
    changed = np.any(dom(R, ur) != dom(R, u0), axis=(0, 2, 3))
    print(lib, "rows changed by do_correct:", np.nonzero(changed)[0])
    assert changed[:2].all() and changed[-2:].all() and not changed[2:-2].any()


@pytest.mark.parametrize("lib,flags", CASES)
def test_steps_from_reference_state(kgpu, oracle, lib, flags):
    if not ref_lib_available(lib):
        pytest.skip(f"{lib} not built")
    R, s = make_pair(kgpu, oracle, lib, 9, flags)
    for step in range(10):
        s.upload_state(R.array("u").copy(), R.array("p").copy())
        s.tstepdenmax = R.scalar("tstepdenmax")
        R.step(1)
        s.rk2_steps(1, graph=step % 2 == 1)
        u, p = s.download_state()
        for tag, a, b in (("u", u, R.array("u")), ("p", p, R.array("p"))):
            ok = close(dom(R, a), dom(R, b), 1e-12)
            assert ok.all(), f"{lib} step {step + 1} {tag}: {np.argwhere(~ok)[:5]}"


def test_radiative_torus_polar_correction(kgpu, oracle):
    if not ref_lib_available(RADLIB):
        pytest.skip(f"{RADLIB} not built")
    R, s = make_pair(kgpu, oracle, RADLIB, 13, 1)
    dt = R.scalar("dt")
    R.L.do_correct()
    R.L.op_explicit(0., dt)
    R.L.calc_u2p()
    s.do_correct()
    s.op_explicit(0., dt)
    s.calc_u2p()
    u, p = s.download_state()
    a, b = dom(R, p), dom(R, R.array("p"))
    mhd = [0, 1, 2, 3, 4, 6, 7, 8]
    assert np.array_equal(a[..., mhd], b[..., mhd])
    assert close(a, b, 1e-11).all()
    assert close(dom(R, u), dom(R, R.array("u")), 1e-12).all()
    # the implicit step leaves the corrected cells as they are
    s.op_implicit(0., dt)
    u2, p2 = s.download_state()
    d, d2 = dom(R, p), dom(R, p2)
    assert np.array_equal(d[:, :2], d2[:, :2]) and np.array_equal(d[:, -2:], d2[:, -2:])
    assert not np.array_equal(d[:, 2:-2], d2[:, 2:-2])
