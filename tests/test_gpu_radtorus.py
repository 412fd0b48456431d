"""CUDA path against the reference KORAL build on the radiative torus: the
magnetised Kerr torus of test_gpu_torus with M1 radiation (RK2IMEX, implicit
lab-frame source solve in every substep, Kramers + electron scattering), on
the small 24x16x8 grid.  As for the MHD torus, the reference computes grid,
metric and initial state; they are uploaded through the C-ABI.

Parity policy.
 - op_explicit: every variable bit-identical except the entropy (CUDA's log
   and pow), held to 1e-12.
 - calc_u2p: MHD variables bit-identical except the entropy; the M1 inversion
   calls pow, so the conserved variables are held to 1e-12 relative and the
   radiation primitives, which the closure's quartic solution amplifies, to
   1e-11 (measured 2.2e-12).
 - op_implicit: the implicit solve of this torus is ill-conditioned (the gas
   energy is the difference of total and radiation energy where radiation
   dominates by up to 1e6), so a last-place difference of pow moves its
   result far more than one ulp.  The reference itself, with the gas energy
   of every cell nudged by one ulp, changes the primitives of most cells;
   the GPU is held to that: per variable, the 90% and 99% quantiles of the
   relative difference within ten times the nudged reference's (plus 1e-13),
   and no more cells whose solve failed than the reference plus a margin.
 - whole steps: the torus is not a smooth map (implicit-solve failures,
   fixups and floors switch branches), so after two steps from the initial
   state the GPU's L1 difference from the reference is held to the largest
   L1 difference the reference itself shows when one input variable of every
   cell is nudged by one ulp (five nudges: gas energy up and down,
   radiation energy up and down, density up), times two.
 - solver variants: the batched and the one-thread-per-cell solvers, and a
   stream and a CUDA-graph replay of the step, give the same bits.
"""
import ctypes
import os
import shutil

import numpy as np
import pytest

from conftest import ref_lib_available

LIB = "libkref_radtorus_small.so"
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_lib_available(LIB), reason="reference radiative torus build not present")]

MASS = 1.e16


def make_gpu(kgpu, R):
    ph = R.physics()
    cfg = kgpu.default_config(R.nx, R.ny, R.nz, ng=R.ng, nv=13, int_order=kgpu.MP5, fluxmethod=kgpu.HLL,
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
    s.set_radiation(kgpu.rad_params(mass=MASS, gamma=ph["gamma"]))
    return s


def second_reference(oracle, tmp_path):
    """An independent instance of the reference build (a copy of the library
    has its own global arrays)."""
    src = os.path.join(oracle.REF_DIR, LIB)
    dst = str(tmp_path / "libkref_radtorus_copy.so")
    shutil.copy(src, dst)
    R = oracle.RefKoral(dst)
    R.init()
    return R


@pytest.fixture(scope="module")
def ref_after_steps(oracle):
    """The reference after three steps, then op_explicit and calc_u2p: the
    states before each operator."""
    R = oracle.RefKoral(LIB)
    R.init()
    R.step(3)
    R.L.op_explicit.argtypes = [ctypes.c_double, ctypes.c_double]
    R.L.op_implicit.argtypes = [ctypes.c_double, ctypes.c_double]
    dt = R.scalar("dt")
    states = {"explicit": (R.array("u").copy(), R.array("p").copy())}
    R.L.op_explicit(0., dt)
    states["explicit_out"] = (R.array("u").copy(), R.array("p").copy())
    R.L.calc_u2p()
    states["u2p_out"] = (R.array("u").copy(), R.array("p").copy())
    return R, dt, states


def dom(R, a):
    g = R.ng
    return a[g:g + R.nz, g:g + R.ny, g:g + R.nx, :]


def close(a, b, rtol):
    scale = np.abs(b).reshape(-1, b.shape[-1]).max(axis=0)
    return np.abs(a - b) <= rtol * (np.abs(b) + 1e-12 * scale)


def test_radtorus_constants_equal_reference(kgpu, oracle):
    R = oracle.RefKoral(LIB)
    c = (ctypes.c_double * 32)()
    R.L.kref_rad_consts(c)
    rp = kgpu.rad_params(mass=MASS, gamma=13.0 / 9.0)
    for i, v in enumerate((rp.kb, rp.mp, rp.sigma, rp.mu, rp.ggg, rp.ccc, rp.masscm)):
        assert v == c[i], i


def test_radtorus_op_explicit_bit_identical(kgpu, ref_after_steps):
    R, dt, st = ref_after_steps
    s = make_gpu(kgpu, R)
    u, p = st["explicit"]
    s.upload_state(u.copy(), p.copy())
    s.op_explicit(0., dt)
    ug, _ = s.download_state()
    a, b = dom(R, ug), dom(R, st["explicit_out"][0])
    others = [v for v in range(13) if v != 5]
    assert np.array_equal(a[..., others], b[..., others])
    assert close(a[..., 5:6], b[..., 5:6], 1e-12).all()


def test_radtorus_calc_u2p_matches_reference(kgpu, ref_after_steps):
    R, dt, st = ref_after_steps
    s = make_gpu(kgpu, R)
    u, p = st["explicit_out"]
    s.upload_state(u.copy(), p.copy())
    s.calc_u2p()
    ug, pg = s.download_state()
    ur, pr = st["u2p_out"]
    a, b = dom(R, pg), dom(R, pr)
    mhd = [0, 1, 2, 3, 4, 6, 7, 8]
    assert np.array_equal(a[..., mhd], b[..., mhd])
    assert close(a, b, 1e-11).all()
    assert close(dom(R, ug), dom(R, ur), 1e-12).all()


def test_radtorus_op_implicit_within_reference_sensitivity(kgpu, oracle, ref_after_steps, tmp_path):
    R, dt, st = ref_after_steps
    gam = 1. - 1. / np.sqrt(2.)
    u, p = st["u2p_out"]
    # the reference, and the reference with the gas energy nudged by one ulp
    R2 = second_reference(oracle, tmp_path)
    R2.L.op_implicit.argtypes = [ctypes.c_double, ctypes.c_double]
    R2.array("u")[...] = u
    R2.array("p")[...] = p
    R2.L.op_implicit(0., dt * gam)
    ref = dom(R2, R2.array("p")).reshape(-1, 13).copy()
    un = u.copy()
    un[..., 1] = np.nextafter(un[..., 1], np.inf)
    R2.array("u")[...] = un
    R2.array("p")[...] = p
    R2.L.op_implicit(0., dt * gam)
    nud = dom(R2, R2.array("p")).reshape(-1, 13).copy()
    s = make_gpu(kgpu, R)
    s.upload_state(u.copy(), p.copy())
    s.reset_counters()
    s.op_implicit(0., dt * gam)
    _, pg = s.download_state()
    gpu = dom(R, pg).reshape(-1, 13)
    c = s.counters()
    assert c["imp_solves"] == gpu.shape[0]
    for v in range(13):
        rg = np.abs(gpu[:, v] - ref[:, v]) / (np.abs(ref[:, v]) + 1e-300)
        rn = np.abs(nud[:, v] - ref[:, v]) / (np.abs(ref[:, v]) + 1e-300)
        for q in (0.9, 0.99):
            a, b = np.quantile(rg, q), np.quantile(rn, q)
            print(f"var {v} q{q}: gpu {a:.2e} nudged reference {b:.2e}")
            assert a <= 10. * b + 1e-13, (v, q, a, b)
    # solves where every attempt failed (RADIMP fixups): a few per cent
    print("GPU failed solves:", c["radimp_failed"])
    assert c["radimp_failed"] <= 0.05 * gpu.shape[0]


def test_radtorus_solver_variants_and_graph_identical(kgpu, oracle):
    R = oracle.RefKoral(LIB)
    R.init()
    u, p, tsd = R.array("u").copy(), R.array("p").copy(), R.scalar("tstepdenmax")
    out = []
    # hard: cells hard in their previous solve start in the tail (0: all that
    # took more than no iteration, i.e. every cell after the first step; -1: none)
    for mode, graph, hard in ((kgpu.RAD_BATCHED, False, 16), (kgpu.RAD_BATCHED, True, 16), (kgpu.RAD_PLAIN, True, 16),
                              (kgpu.RAD_PERSISTENT, False, 16), (kgpu.RAD_PERSISTENT, True, 16),
                              (kgpu.RAD_BATCHED, True, -1), (kgpu.RAD_BATCHED, True, 0)):
        s = make_gpu(kgpu, R)
        s.set_implicit_solver(mode, None)
        s.set_implicit_options(hard=hard)
        s.upload_state(u.copy(), p.copy())
        s.tstepdenmax = tsd
        s.rk2imex_steps(3, graph=graph)
        out.append(s.download_state())
        s.close()
    for k in range(1, len(out)):
        assert np.array_equal(out[0][0], out[k][0]) and np.array_equal(out[0][1], out[k][1]), k


def test_radtorus_solver_options_per_context(kgpu, oracle):
    """Two contexts in one process hold their own solver tuning: setting one
    leaves the other alone, a captured step graph is re-captured when its
    context's options change (its launch count follows them), and the
    results stay the same bits."""
    R = oracle.RefKoral(LIB)
    R.init()
    u, p, tsd = R.array("u").copy(), R.array("p").copy(), R.scalar("tstepdenmax")
    a, b = make_gpu(kgpu, R), make_gpu(kgpu, R)
    for s in (a, b):
        s.set_implicit_solver(kgpu.RAD_BATCHED, None)
        s.upload_state(u.copy(), p.copy())
        s.tstepdenmax = tsd
    a.set_implicit_options(pass_iters=1)
    assert b.implicit_options().pass_iters == kgpu.solver_opts().pass_iters and a.implicit_options().pass_iters == 1
    la = a.launches
    a.rk2imex_steps(1, graph=True)
    la = a.launches - la
    lb = b.launches
    b.rk2imex_steps(1, graph=True)
    lb = b.launches - lb
    assert la > lb   # one Newton iteration per pass: more pass launches
    b.set_implicit_options(pass_iters=1)   # between two graph steps: re-captured
    lb2 = b.launches
    b.rk2imex_steps(1, graph=True)
    assert b.launches - lb2 == la
    a.rk2imex_steps(1, graph=True)
    ua, pa = a.download_state()
    ub, pb = b.download_state()
    assert np.array_equal(ua, ub) and np.array_equal(pa, pb)
    with pytest.raises(kgpu.KgpuError):
        a.set_implicit_options(thin=33)


def test_radtorus_two_steps_within_reference_sensitivity(kgpu, oracle, tmp_path):
    """Two whole RK2IMEX steps from the initial state: the GPU against the
    reference, measured against the spread of the reference's own one-ulp
    nudges."""
    R = oracle.RefKoral(LIB)
    R.init()
    u, p, tsd = R.array("u").copy(), R.array("p").copy(), R.scalar("tstepdenmax")
    s = make_gpu(kgpu, R)
    s.upload_state(u.copy(), p.copy())
    s.tstepdenmax = tsd
    R.step(2)
    s.rk2imex_steps(2)
    ref = dom(R, R.array("u")).reshape(-1, 13)
    ug, _ = s.download_state()
    gpu = dom(R, ug).reshape(-1, 13)
    assert abs(s.tstepdenmax - R.scalar("tstepdenmax")) <= 1e-8 * R.scalar("tstepdenmax")

    def l1(a):
        return np.array([np.abs(a[:, v] - ref[:, v]).sum() / (np.abs(ref[:, v]).sum() + 1e-300) for v in range(13)])

    spread = np.zeros(13)
    for j, (var, direction) in enumerate(((1, np.inf), (1, -np.inf), (9, np.inf), (9, -np.inf), (0, np.inf))):
        src = os.path.join(oracle.REF_DIR, LIB)
        dst = str(tmp_path / f"libkref_radtorus_nudge{j}.so")
        shutil.copy(src, dst)
        N = oracle.RefKoral(dst)
        N.init()
        N.array("u")[..., var] = np.nextafter(N.array("u")[..., var], direction)
        N.step(2)
        spread = np.maximum(spread, l1(dom(N, N.array("u")).reshape(-1, 13)))
    got = l1(gpu)
    for v in range(13):
        print(f"var {v}: L1 gpu {got[v]:.2e} largest one-ulp nudge of the reference {spread[v]:.2e}")
        assert got[v] <= 2. * spread[v] + 1e-12, (v, got[v], spread[v])
