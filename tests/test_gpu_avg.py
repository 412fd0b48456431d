"""Time averages (save_avg, fileop.c:10-70, of the quantities of p2avg,
p2u.c:313-541) on the device against the reference build's own save_avg.

Both sides start from the reference's state after a few steps and run
op_explicit (which leaves the primitives as they were and the face fluxes
after flux_ct), then save_avg(dt) into zeroed sums.  Every slot is
bit-identical except those that go through the host C library's pow or
log on the reference side: the entropy's face flux (the face floors
recompute the entropy) and, with radiation, the fluid-frame four-force
(Planck term and Kramers opacity); those agree to 1e-12 relative.  Two
slots the reference never sets (an uninitialised local array there) are
left out: AVGEHAT without radiation and AVGGHATCOMPT.

The fused steps call save_avg once per step where the reference's loop
does; for RK2 that point is after the second stage's inversion, whose
primitives and face fluxes the step leaves in place, so one fused step
with the averages on equals the same step followed by kgpu_save_avg.
"""
import ctypes

import numpy as np
import pytest

from conftest import ref_lib_available

pytestmark = pytest.mark.gpu

TORUS = "libkref_fmtorus_small.so"
RADTORUS = "libkref_radtorus_small.so"


def make_pair(kgpu, oracle, lib, nv):
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
    s.upload_state(R.array("u").copy(), R.array("p").copy())
    s.tstepdenmax = R.scalar("tstepdenmax")
    return R, s


def slots(nv, rad):
    """(number of slots, slots left out, slots through pow/log)"""
    navg = (153 if rad else 112) + 3 * nv
    skip = [4 * nv + 148 + i for i in range(4)] if rad else [4 * nv + 111]
    libm = [nv + 109 + 5, nv + 109 + nv + 5, nv + 109 + 2 * nv + 5]   # entropy fluxes at the three left faces
    if rad:
        libm += [4 * nv + 144 + i for i in range(4)]                   # AVGGHAT
    return nv + navg, skip, libm


@pytest.mark.parametrize("lib,nv", [(TORUS, 9), (RADTORUS, 13)])
def test_save_avg_matches_reference(kgpu, oracle, lib, nv):
    if not ref_lib_available(lib):
        pytest.skip(f"{lib} not built")
    R, s = make_pair(kgpu, oracle, lib, nv)
    nav, skip, libm = slots(nv, nv == 13)
    dt = R.scalar("dt")
    R.L.op_explicit(0., dt)
    s.op_explicit(0., dt)
    pref = R.array("pavg", (R.sz, R.sy, R.sx, nav))
    pref[...] = 0.
    R.set_scalar("avgtime", 0.)
    R.L.save_avg.argtypes = [ctypes.c_double]
    R.L.save_avg(dt)
    s.set_avg(on=False, mass=10.0)
    s.save_avg(dt)
    got, t = s.download_avg()
    assert got.shape[-1] == nav
    assert t == R.scalar("avgtime") == dt
    g = R.ng
    a = got[g:g + R.nz, g:g + R.ny, g:g + R.nx].reshape(-1, nav)
    b = pref[g:g + R.nz, g:g + R.ny, g:g + R.nx].reshape(-1, nav)
    keep = [i for i in range(nav) if i not in skip]
    exact = [i for i in keep if i not in libm]
    diff = [i for i in exact if not np.array_equal(a[:, i], b[:, i])]
    assert not diff, f"slots not bit-identical: {diff}"
    scale = np.abs(b).max(axis=0)
    rel = np.abs(a[:, libm] - b[:, libm]) / (np.abs(b[:, libm]) + 1e-6 * scale[libm] + 1e-300)
    print(f"{lib}: {len(exact)} slots bit-identical, {len(libm)} through pow/log within {rel.max():.2e}")
    assert rel.max() <= 1e-12
    assert np.all(np.isfinite(a[:, keep]))
    assert np.all(got[:g] == 0.)   # ghost cells untouched


def test_fused_rk2_step_saves_averages_once(kgpu, oracle):
    if not ref_lib_available(TORUS):
        pytest.skip(f"{TORUS} not built")
    R, s = make_pair(kgpu, oracle, TORUS, 9)
    u0, p0 = R.array("u").copy(), R.array("p").copy()
    td = R.scalar("tstepdenmax")
    s.set_avg(on=True, mass=10.0)
    s.rk2_steps(1, graph=True)
    a1, t1 = s.download_avg()
    assert t1 == 1. / td
    # the same step without the averages, then save_avg with its dt
    s.set_avg(on=False)
    s.reset_avg()
    s.upload_state(u0, p0)
    s.tstepdenmax = td
    s.rk2_steps(1, graph=False)
    s.save_avg(1. / td)
    a2, t2 = s.download_avg()
    assert t2 == t1 and np.array_equal(a1, a2)
    # two graph steps with the averages on add both time steps
    s.set_avg(on=True)
    s.reset_avg()
    s.upload_state(u0, p0)
    s.tstepdenmax = td
    s.rk2_steps(1, graph=True)
    td2 = s.tstepdenmax
    s.rk2_steps(1, graph=True)
    _, t3 = s.download_avg()
    assert t3 == (0. + 1. / td) + 1. / td2


def test_fused_rk2imex_step_saves_averages(kgpu, oracle):
    if not ref_lib_available(RADTORUS):
        pytest.skip(f"{RADTORUS} not built")
    R, s = make_pair(kgpu, oracle, RADTORUS, 13)
    td = R.scalar("tstepdenmax")
    s.set_avg(on=True)
    s.rk2imex_steps(1, graph=True)
    a, t = s.download_avg()
    assert t == 1. / td
    g, nv = R.ng, 13
    d = a[g:g + R.nz, g:g + R.ny, g:g + R.nx].reshape(-1, a.shape[-1])
    nav, skip, _ = slots(nv, True)
    keep = [i for i in range(nav) if i not in skip]
    assert np.all(np.isfinite(d[:, keep]))
    # averaged density and fluid-frame radiation energy are positive
    assert np.all(d[:, 0] > 0.) and np.all(d[:, 4 * nv + 111] > 0.)
