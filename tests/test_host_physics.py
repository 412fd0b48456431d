"""The library's per-cell physics, compiled for the host from the same
headers the kernels are built from (koral_b200/csrc/kgpu_physics.cuh,
kgpu_rad.cuh; harness tests/hostphys/physics_host.cu), against the oracle
and the reference build on the CPU.  The host build rounds +, -, *, /, sqrt
as the device build does (no FMA contraction, IEEE division and square
root) and calls the host C library's log and pow where the device calls
CUDA's, so it shows, without a GPU, that the source restates the reference
operation for operation:

* MHD, at metric points of the Kerr torus: p2u, the three flux rows, the
  wave speeds, the inversion (u2p.c:176, energy and entropy equations and
  the failure path), the floors with the magnetisation ceiling at 100 and
  at 0.3; the inversion in flat spacetime up to Lorentz factors of a few
  hundred; PPM and MP5 reconstruction: bit for bit against the oracle.
* Radiation, on cells of the batched implicit-solve workload: p2u of the 13
  variables and the M1 inversion (with superluminal fluxes and negative
  energies, which take its corrections) bit for bit against the reference
  build;
  the implicit source solve (rad.c:1225-1570) equal to the reference's in
  every cell once the solver's two own powers (T^4 of the Planck term and
  the squares of the M1 closure, double-double products rounded once) are
  replaced by the C library's pow, and with them equal in status in every
  cell and bit for bit in 99% of cells; where it differs, it does by less
  than ten times the reference's own sensitivity to a one-ulp nudge of its
  input.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, ref_lib_available

HARNESS = os.path.join(ROOT, "tests", "hostphys", "physics_host.cu")
CSRC = os.path.join(ROOT, "koral_b200", "csrc")
LIBDIR = os.path.join(ROOT, "koral_b200", "_lib")
NVCC = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O2", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-diag-suppress", "550", "-shared"]
# the solver's own powers, and the C library's pow in their place
LIBM_POWERS = [("R.sigma * pw4(Tgas)", "R.sigma * pow(Tgas, 4.)"),
               ("KG_HD double m1_pow2(double x) { return pw2(x); }",
                "KG_HD double m1_pow2(double x) { return pow(x, 2.); }")]

pytestmark = pytest.mark.skipif(NVCC is None, reason="nvcc not present")

dp = ctypes.POINTER(ctypes.c_double)
ip = ctypes.POINTER(ctypes.c_int)


def P(a):
    return a.ctypes.data_as(dp)


def I(a):
    return a.ctypes.data_as(ip)


def compile_harness(out, src):
    subprocess.check_call([NVCC] + FLAGS + ["-o", out, src, "-L", LIBDIR, "-lkoral_b200", "-Xlinker",
                                            "-rpath=" + LIBDIR])
    return ctypes.CDLL(out)


@pytest.fixture(scope="module")
def host(kgpu, tmp_path_factory):
    return compile_harness(str(tmp_path_factory.mktemp("hostphys") / "libhostphys.so"), HARNESS)


@pytest.fixture(scope="module")
def host_libm(kgpu, tmp_path_factory):
    """The same harness over a copy of the headers whose two powers call the
    C library's pow."""
    d = tmp_path_factory.mktemp("hostphys_libm")
    (d / "koral_b200" / "csrc").mkdir(parents=True)
    (d / "include").mkdir()
    (d / "tests" / "hostphys").mkdir(parents=True)
    for f in os.listdir(CSRC):
        if f.endswith(".cuh"):
            shutil.copy(os.path.join(CSRC, f), d / "koral_b200" / "csrc" / f)
    shutil.copy(os.path.join(ROOT, "include", "koral_b200.h"), d / "include")
    shutil.copy(HARNESS, d / "tests" / "hostphys")
    rad = d / "koral_b200" / "csrc" / "kgpu_rad.cuh"
    text = rad.read_text()
    for old, new in LIBM_POWERS:
        assert text.count(old) == 1, old
        text = text.replace(old, new)
    rad.write_text(text)
    return compile_harness(str(d / "libhostphys_libm.so"), str(d / "tests" / "hostphys" / "physics_host.cu"))


class KoGeom(ctypes.Structure):
    _fields_ = [("gg", ctypes.c_double * 20), ("GG", ctypes.c_double * 20), ("gdet", ctypes.c_double),
                ("gttpert", ctypes.c_double), ("alpha", ctypes.c_double)]


@pytest.fixture(scope="module")
def torus_cells(oracle):
    """20000 magnetised states at metric points of the small torus's grid."""
    if not ref_lib_available("libkref_fmtorus_small.so"):
        pytest.skip("reference torus build not present")
    R = oracle.RefKoral("libkref_fmtorus_small.so")
    R.init()
    g, G = R.metric_tables()[:2]
    g, G = g.reshape(-1, 20), G.reshape(-1, 20)
    ok = np.isfinite(g).all(axis=1) & (g[:, 19] > 0)
    g, G = g[ok], G[ok]
    rng = np.random.default_rng(3)
    n = 20000
    idx = rng.integers(0, len(g), n)
    gm, Gm = np.ascontiguousarray(g[idx]), np.ascontiguousarray(G[idx])
    gam = R.physics()["gamma"]
    pp = np.zeros((n, 9))
    pp[:, 0] = 10 ** rng.uniform(-5, 0, n)
    pp[:, 1] = pp[:, 0] * 10 ** rng.uniform(-4, 1, n)
    pp[:, 2:5] = rng.normal(0, 0.5, (n, 3))
    pp[:, 6:9] = rng.normal(0, 1.0, (n, 3)) * np.sqrt(pp[:, :1]) * 10 ** rng.uniform(-1.5, 1, (n, 1))
    pp[:, 5] = pp[:, 0] * np.log(((gam - 1) * pp[:, 1]) ** (1 / (gam - 1)) / pp[:, 0] ** (1 / (gam - 1) + 1))
    O = oracle.OracleGrid(8, 8, 1, 3, 9)
    O.set_physics(gam, 0.5, 4, 1)
    return O, gam, pp, gm, Gm, rng


def test_mhd_point_physics_bit_identical(host, torus_cells):
    O, gam, pp, gm, Gm, _ = torus_cells
    n = pp.shape[0]
    L = O.lib()
    L.ko_flux_prime.argtypes = [ctypes.c_void_p, dp, ctypes.c_int, ctypes.POINTER(KoGeom), dp]
    L.ko_wavespeeds_lr_pure.argtypes = [ctypes.c_void_p, dp, ctypes.POINTER(KoGeom), dp]
    out = np.zeros((n, 9))
    host.hp_mhd_point(ctypes.c_long(n), 0, ctypes.c_double(gam), P(pp), P(gm), P(Gm), P(out))
    assert np.array_equal(out, O.p2u_batch(pp, gm, Gm))
    m = 4000   # the oracle's per-point routines, one call per cell
    geoms = []
    for i in range(m):
        k = KoGeom()
        k.gg[:] = list(gm[i])
        k.GG[:] = list(Gm[i])
        k.alpha, k.gdet, k.gttpert = np.sqrt(-1. / Gm[i, 0]), gm[i, 19], Gm[i, 19]
        geoms.append(k)
    rows = [np.ascontiguousarray(pp[i]) for i in range(m)]
    for d in range(3):
        ref = np.zeros((m, 9))
        for i in range(m):
            L.ko_flux_prime(O.h, P(rows[i]), d, ctypes.byref(geoms[i]), P(ref[i]))
        host.hp_mhd_point(ctypes.c_long(n), d + 1, ctypes.c_double(gam), P(pp), P(gm), P(Gm), P(out))
        assert np.array_equal(out[:m], ref), f"flux row {d}"
    ref = np.zeros((m, 12))
    for i in range(m):
        L.ko_wavespeeds_lr_pure(O.h, P(rows[i]), ctypes.byref(geoms[i]), P(ref[i]))
    ws = np.zeros((n, 6))
    host.hp_mhd_point(ctypes.c_long(n), 4, ctypes.c_double(gam), P(pp), P(gm), P(Gm), P(ws))
    assert np.array_equal(ws[:m], ref[:, :6])


def test_mhd_inversion_and_floors_bit_identical(host, torus_cells):
    O, gam, pp, gm, Gm, rng = torus_cells
    n = pp.shape[0]
    O.set_floors(1e-50, 1e-50, 100., 100., 100.)
    uu = O.p2u_batch(pp, gm, Gm)
    guess = pp * (1 + rng.uniform(-0.1, 0.1, pp.shape))
    po, so, fo = O.u2p_batch(uu, guess, gm, Gm)
    ph, rh, fh = guess.copy(), np.zeros(n, np.int32), np.zeros(n, np.int32)
    host.hp_u2p(ctypes.c_long(n), 0, ctypes.c_double(gam), ctypes.c_double(100.), P(uu), P(ph), P(gm), P(Gm), I(rh),
                I(fh))
    kinds = dict(zip(*np.unique(so, return_counts=True)))
    print("inversion statuses (0 energy, -1 entropy, -3 failed):", kinds)
    assert kinds.get(-1, 0) > 0 and kinds.get(-3, 0) > 0
    assert np.array_equal(rh, so) and np.array_equal(fh, fo) and np.array_equal(ph, po)
    for b2rho in (100., 0.3):
        O.set_floors(1e-50, 1e-50, 100., b2rho, 100.)
        a, ra = pp.copy(), np.zeros(n, np.int32)
        O.lib().ko_floors_batch(ctypes.c_void_p(O.h), n, P(a), P(gm), P(Gm), I(ra))
        b, rb, fx = pp.copy(), np.zeros(n, np.int32), np.zeros(n, np.int32)
        host.hp_u2p(ctypes.c_long(n), 1, ctypes.c_double(gam), ctypes.c_double(b2rho), None, P(b), P(gm), P(Gm),
                    I(rb), I(fx))
        print(f"floors, ceiling {b2rho}: acted in {np.mean(ra != 0):.3f} of the states")
        assert np.mean(ra != 0) > 0.5
        assert np.array_equal(ra, rb) and np.array_equal(a, b)


@pytest.mark.parametrize("vscale", [2., 10., 50.])
def test_mhd_inversion_flat_high_lorentz_bit_identical(host, oracle, vscale):
    """Flat spacetime, spatial four-velocity components of scale vscale
    (Lorentz factors up to a few hundred at 50)."""
    rng = np.random.default_rng(int(vscale))
    n = 20000
    g, G = np.zeros((n, 20)), np.zeros((n, 20))
    for a, v in ((0, -1.), (6, 1.), (12, 1.), (18, 1.), (19, 1.)):
        g[:, a] = v
    for a, v in ((0, -1.), (6, 1.), (12, 1.), (18, 1.)):
        G[:, a] = v
    pp = np.zeros((n, 9))
    pp[:, 0] = 10 ** rng.uniform(-4, 1, n)
    pp[:, 1] = pp[:, 0] * 10 ** rng.uniform(-4, 1.5, n)
    pp[:, 2:5] = rng.normal(0, vscale, (n, 3))
    pp[:, 6:9] = rng.normal(0, 1, (n, 3)) * np.sqrt(pp[:, :1]) * 10 ** rng.uniform(-2, 1, (n, 1))
    pp[:, 5] = pp[:, 0] * np.log(((2 / 3) * pp[:, 1]) ** 1.5 / pp[:, 0] ** 2.5)
    O = oracle.OracleGrid(8, 8, 1, 3, 9)
    O.set_physics(5. / 3., 0.5, 2, 0)
    uu = O.p2u_batch(pp, g, G)
    guess = pp * (1 + rng.uniform(-0.1, 0.1, pp.shape))
    po, so, fo = O.u2p_batch(uu, guess, g, G)
    ph, rh, fh = guess.copy(), np.zeros(n, np.int32), np.zeros(n, np.int32)
    host.hp_u2p(ctypes.c_long(n), 0, ctypes.c_double(5. / 3.), ctypes.c_double(100.), P(uu), P(ph), P(g), P(G), I(rh),
                I(fh))
    assert np.array_equal(rh, so) and np.array_equal(fh, fo) and np.array_equal(ph, po)


@pytest.mark.parametrize("order", [2, 4])
def test_reconstruction_bit_identical(host, oracle, order):
    rng = np.random.default_rng(order)
    O = oracle.OracleGrid(8, 8, 1, 3, 9)
    O.set_physics(13. / 9., 0.5, order, 1)
    L = O.lib()
    L.ko_avg2point.argtypes = [ctypes.c_void_p] + [dp] * 7 + [ctypes.c_double] * 5
    k = 9 * 1000
    u = rng.normal(size=(k, 5)) * 10 ** rng.uniform(-3, 3, (k, 1)) + rng.normal(size=(k, 1))
    u[::7, 3] = u[::7, 2]   # flat pieces and extrema
    u[::11, 1] = u[::11, 3]
    dx = np.repeat(10 ** rng.uniform(-2, 0, (k // 9, 5)), 9, axis=0) if order == 2 else np.ones((k, 5))
    left, right = np.zeros(k), np.zeros(k)
    for c in range(0, k, 9):   # nine stencils per call, as the nine variables of one face
        cols = [np.ascontiguousarray(u[c:c + 9, j]) for j in range(5)]
        L.ko_avg2point(O.h, P(cols[0]), P(cols[1]), P(cols[2]), P(cols[3]), P(cols[4]), P(left[c:]),
                       P(right[c:]), *[float(x) for x in dx[c]])
    lh, rh = np.zeros(k), np.zeros(k)
    host.hp_recon(ctypes.c_long(k), order, P(np.ascontiguousarray(u)), P(np.ascontiguousarray(dx)), P(lh), P(rh))
    assert np.array_equal(lh, left) and np.array_equal(rh, right)


@pytest.fixture(scope="module")
def rad_cells(kgpu, oracle):
    if not ref_lib_available("libkref_radcells.so"):
        pytest.skip("reference radiating-cells build not present")
    ref = oracle.RefRadCells()
    rp = kgpu.rad_params()
    pp, g, G, tau = kgpu.rad_cell_draws(4096, 2026, rp, metric=ref.metric)
    uu, kabs, kes = ref.prepare(pp, g, G)
    dt = 0.5 * tau / (kabs + kes)
    return ref, rp, uu, pp, g, G, dt


def test_rad_p2u_and_m1_inversion_bit_identical(host, rad_cells):
    ref, rp, uu, pp, g, G, dt = rad_cells
    n = uu.shape[0]
    out = np.zeros_like(pp)
    host.hp_rad_cells(ctypes.c_long(n), 0, ctypes.byref(rp), P(uu), P(pp), P(g), P(G), P(out), None, None)
    assert np.array_equal(out, uu)
    guess = pp.copy()
    guess[:, 9:] *= 0.9
    half = np.arange(n) % 2 == 0
    for case in ("plain", "flux above the energy", "negative energy"):
        u = uu.copy()
        if case == "flux above the energy":
            u[half, 10:13] *= 3.
        elif case == "negative energy":
            u[half, 9] *= -1e-3
        pr, sr, cr = ref.u2p(u, guess, g, G)
        ph, sh, ch = guess.copy(), np.zeros(n, np.int32), np.zeros(n, np.int32)
        host.hp_rad_cells(ctypes.c_long(n), 1, ctypes.byref(rp), P(u), P(ph), P(g), P(G), None, I(sh), I(ch))
        print(f"M1 inversion, {case}: {int(cr.sum())} corrected")
        assert case == "plain" or cr.sum() > 0
        assert np.array_equal(sh, sr) and np.array_equal(ch, cr) and np.array_equal(ph, pr), case


def solve(lib, rp, uu, pp, g, G, dt):
    n = uu.shape[0]
    po, uo = np.zeros_like(pp), np.zeros_like(uu)
    st, at, it = (np.zeros(n, np.int32) for _ in range(3))
    lib.hp_rad_implicit(ctypes.c_long(n), ctypes.byref(rp), P(uu), P(pp), P(g), P(G), P(dt), P(po), P(uo), I(st),
                        I(at), I(it))
    return po, uo, st, at, it


def test_rad_implicit_solve_matches_reference(host, host_libm, rad_cells):
    from test_gpu_rad import scaled_difference
    ref, rp, uu, pp, g, G, dt = rad_cells
    pr, ur, sr, wr, ir = ref.implicit(uu, pp, g, G, dt)
    # with the C library's pow in place of the solver's own powers: every
    # cell, every bit
    pl, ul, sl, al, il = solve(host_libm, rp, uu, pp, g, G, dt)
    assert np.array_equal(sl, sr) and np.array_equal(il, ir) and np.array_equal(pl, pr) and np.array_equal(ul, ur)
    # the product's source as it is
    ph, uh, sh, ah, ih = solve(host, rp, uu, pp, g, G, dt)
    same = np.all(ph == pr, axis=1) & np.all(uh == ur, axis=1)
    print(f"implicit solve, host build of the product source: {np.mean(same):.4f} of cells bit-identical, "
          f"{int(np.sum(sr != 0))} failed solves in both")
    assert np.array_equal(sh, sr)
    assert np.mean(same) >= 0.99
    un = uu.copy()
    un[:, 1] = np.nextafter(un[:, 1], np.inf)
    pn, _, sn, _, _ = ref.implicit(un, pp, g, G, dt)
    q = [0.5, 0.9, 0.99]
    both, bn = (sh == 0) & (sr == 0), (sn == 0) & (sr == 0)
    dh = np.quantile(scaled_difference(ph[both], pr[both]), q)
    dn = np.quantile(scaled_difference(pn[bn], pr[bn]), q)
    assert np.all(dh <= 10 * dn + 1e-12), (dh, dn)
