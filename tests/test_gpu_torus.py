"""CUDA path against the reference KORAL build on the magnetised Kerr torus
(MKS2, spin 0.9, MP5 + HLL + flux-CT, torus boundaries, radius-dependent
density floor) on a small 24x16x8 grid.

The host side is used exactly as a drop-in: the reference computes the grid,
the metric tables (calc_metric) and the initial state on the CPU; they are
uploaded through the C-ABI and the device runs the operators.

Tolerance: per step, conserved variables must agree to 1e-12 relative
(|a-b| <= 1e-12 (|b| + 1e-6 max|b_v|)); in practice all but the entropy are
bit-identical.  After 100 free-running steps the L1 difference is held to
the reference's own drift under a one-ulp nudge (see the free-run test).
"""
import numpy as np
import pytest

from conftest import ref_lib_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_lib_available("libkref_fmtorus_small.so"),
                                 reason="reference torus build not present")]

LIB = "libkref_fmtorus_small.so"


def make_pair(kgpu, oracle):
    R = oracle.RefKoral(LIB)
    R.init()
    ph = R.physics()
    cfg = kgpu.default_config(R.nx, R.ny, R.nz, ng=R.ng, int_order=kgpu.MP5, fluxmethod=kgpu.HLL,
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
    s.upload_state(R.array("u").copy(), R.array("p").copy())
    s.tstepdenmax = R.scalar("tstepdenmax")
    return R, s


def dom(R, a):
    g = R.ng
    return a[g:g + R.nz, g:g + R.ny, g:g + R.nx, :]


def check_close(R, got, ref, tag, rtol=1e-12):
    g, r = dom(R, got), dom(R, ref)
    scale = np.abs(r).reshape(-1, r.shape[-1]).max(axis=0)
    bad = np.abs(g - r) > rtol * (np.abs(r) + 1e-6 * scale)
    assert not bad.any(), f"{tag}: {bad.sum()} values beyond tolerance, vars {np.unique(np.argwhere(bad)[:, -1])}"
    return np.count_nonzero(g[..., [0, 1, 2, 3, 4, 6, 7, 8]] != r[..., [0, 1, 2, 3, 4, 6, 7, 8]])


def test_torus_single_steps_from_reference_state(kgpu, oracle):
    """Each of 100 steps starts from the reference's state (re-uploaded), so
    every step of the reference's trajectory is checked on its own."""
    R, s = make_pair(kgpu, oracle)
    ndiff = 0
    for step in range(100):
        s.upload_state(R.array("u").copy(), R.array("p").copy())
        s.tstepdenmax = R.scalar("tstepdenmax")
        R.step(1)
        s.rk2_steps(1)
        u, p = s.download_state()
        ndiff += check_close(R, u, R.array("u"), f"u step {step + 1}")
        ndiff += check_close(R, p, R.array("p"), f"p step {step + 1}")
        assert s.tstepdenmax == R.scalar("tstepdenmax") or \
            abs(s.tstepdenmax - R.scalar("tstepdenmax")) <= 1e-12 * R.scalar("tstepdenmax")
    print("values not bit-identical (non-entropy):", ndiff)


def l1_rel(a, b):
    """L1 difference per conserved variable, normalised by b's L1 norm; the
    three momentum components share one scale, the largest of their norms,
    because the theta-momentum of a torus near equilibrium is close to zero
    and its own norm says little."""
    norm = np.abs(b).sum(axis=(0, 1, 2))
    norm[2:5] = norm[2:5].max()
    return np.abs(a - b).sum(axis=(0, 1, 2)) / norm.clip(1e-300)


# cells inside the torus (z, y, x, var) whose energy gets a one-ulp nudge
NUDGED = [(4, 8, 6, 1), (2, 7, 8, 1), (6, 9, 5, 1)]


def test_torus_free_run_l1(kgpu, oracle):
    """100 free-running RK2 steps, against the reference's own sensitivity.

    This torus is not smooth in the reference either: floors, fixups and
    inversion failures switch branches, and the reference run with the
    energy of a single cell changed by one ulp drifts from the unperturbed
    run to a relative L1 of about 1e-5 in density (1e-3 in entropy) after
    100 steps.  The GPU's entropy inversion uses CUDA's log and pow, whose
    last-place results differ from the host library's, so after 100 steps
    the two can only be expected to agree as well as the reference agrees
    with itself under a one-ulp nudge.  Bar: per variable, the GPU's L1
    difference is at most ten times the largest drift of the reference over
    three one-ulp nudges.  A genuine defect moves L1 to 1e-2 or more."""
    R, s = make_pair(kgpu, oracle)
    R.step(100)
    ref = dom(R, R.array("u")).copy()
    s.rk2_steps(100, graph=True)
    u, _ = s.download_state()
    got = dom(R, u)
    assert np.isfinite(got).all()
    l1 = l1_rel(got, ref)
    drift = np.zeros(9)
    for cell in NUDGED:
        R.init()
        a = R.array("u")
        c = (cell[0] + R.ng, cell[1] + R.ng, cell[2] + R.ng, cell[3])
        a[c] = np.nextafter(a[c], np.inf)
        R.step(100)
        drift = np.maximum(drift, l1_rel(dom(R, R.array("u")), ref))
    print("GPU vs reference, relative L1 after 100 steps:", l1)
    print("reference vs one-ulp nudged reference:        ", drift)
    assert (drift > 0).all()
    assert (l1 <= 10 * drift).all(), (l1, drift)


def test_u2p_at_kerr_points_matches_oracle(kgpu, oracle):
    """Batched inversion at metric points of the MKS2 Kerr grid (non-trivial
    g_ti, lapse and shift) against the C restatement."""
    R = oracle.RefKoral(LIB)
    R.init()
    g, G = R.metric_tables()[:2]
    g = g.reshape(-1, 20)
    G = G.reshape(-1, 20)
    ok = np.isfinite(g).all(axis=1) & (g[:, 19] > 0)
    g, G = g[ok], G[ok]
    rng = np.random.default_rng(5)
    n = 20000
    idx = rng.integers(0, len(g), n)
    gm, Gm = g[idx].copy(), G[idx].copy()
    pp = np.zeros((n, 9))
    pp[:, 0] = 10 ** rng.uniform(-5, 0, n)
    pp[:, 1] = pp[:, 0] * 10 ** rng.uniform(-4, 1, n)
    pp[:, 2:5] = rng.normal(0, 0.5, (n, 3))
    pp[:, 6:9] = rng.normal(0, 0.1, (n, 3)) * np.sqrt(pp[:, :1])
    gam = R.physics()["gamma"]
    pp[:, 5] = pp[:, 0] * np.log(((gam - 1) * pp[:, 1]) ** (1 / (gam - 1)) / pp[:, 0] ** (1 / (gam - 1) + 1))
    Og = oracle.OracleGrid(8, 8, 1, 3, 9)
    Og.set_physics(gam, 0.5, 4, 1)
    cfg = kgpu.default_config(8, 8, 1, gamma=gam)
    uu = Og.p2u_batch(pp, gm, Gm)
    assert np.array_equal(kgpu.p2u_cells(cfg, pp, gm, Gm)[:, [0, 1, 2, 3, 4, 6, 7, 8]], uu[:, [0, 1, 2, 3, 4, 6, 7, 8]])
    guess = pp * (1 + rng.uniform(-0.05, 0.05, pp.shape))
    po, so, fo = Og.u2p_batch(uu, guess, gm, Gm)
    pg, sg, fg = kgpu.u2p_cells(cfg, uu, guess, gm, Gm)
    assert np.array_equal(sg, so) and np.array_equal(fg, fo)
    hot = so == 0
    assert hot.mean() > 0.9
    assert np.array_equal(pg[hot][:, [0, 1, 2, 3, 4, 6, 7, 8]], po[hot][:, [0, 1, 2, 3, 4, 6, 7, 8]])


def test_u2p_pause_and_resume_is_exact(kgpu, oracle):
    """The inversion runs as passes over work queues: a cell whose Newton
    solve is not done after a few steps, or needs many damping halvings, is
    paused and resumed in a later pass (one warp per cell).  Where the pause
    falls must not change any bit of the result."""
    R, s = make_pair(kgpu, oracle)
    u0, p0 = R.array("u").copy(), R.array("p").copy()
    tsd = R.scalar("tstepdenmax")
    states = []
    for n in (8, 1, 3, 1000):
        s.upload_state(u0.copy(), p0.copy())
        s.tstepdenmax = tsd
        s.set_u2p_pass_iters(n)
        s.reset_counters()
        s.rk2_steps(20)
        states.append(s.download_state())
        cnt = s.counters()
        if n == 1:
            assert cnt["paused"] > 0
        print(f"pass limit {n}: faces whose state needed the magnetic floor over 20 steps: {cnt['face_floors']}")
    for u, p in states[1:]:
        assert np.array_equal(u, states[0][0]) and np.array_equal(p, states[0][1])


def test_flux_ct_fluxes_match_reference(kgpu, oracle):
    """flux_ct through the C-ABI: after op_explicit from the reference's
    state, kgpu_flux_ct stores the face fluxes with their magnetic
    components rewritten from the corner EMFs; they equal the reference's
    flbx/flby/flbz after its op_explicit (which calls flux_ct), every
    variable bit for bit except the entropy flux (1e-12).  A second call
    for the same op_explicit is refused."""
    R, s = make_pair(kgpu, oracle)
    R.step(3)
    s.upload_state(R.array("u").copy(), R.array("p").copy())
    s.tstepdenmax = R.scalar("tstepdenmax")
    import ctypes
    R.L.op_explicit.argtypes = [ctypes.c_double, ctypes.c_double]
    dt = R.scalar("dt")
    R.L.op_explicit(0., dt)
    s.op_explicit(0., dt)
    s.flux_ct()
    with pytest.raises(kgpu.KgpuError):
        s.flux_ct()
    g, nx, ny, nz, nv = R.ng, R.nx, R.ny, R.nz, R.nv
    sx, sy, sz = R.sx, R.sy, R.sz
    shapes = {0: ("flbx", (sz, sy, sx + 1, nv), (nz, ny, nx + 1)), 1: ("flby", (sz, sy + 1, sx, nv), (nz, ny + 1, nx)),
              2: ("flbz", (sz + 1, sy, sx, nv), (nz + 1, ny, nx))}
    for d, (name, shp, (kz, ky, kx)) in shapes.items():
        got = s.download_flux(d).reshape(shp)[g:g + kz, g:g + ky, g:g + kx]
        ref = R.array(name, shp)[g:g + kz, g:g + ky, g:g + kx]
        nonent = [0, 1, 2, 3, 4, 6, 7, 8]
        assert np.array_equal(got[..., nonent], ref[..., nonent]), name
        assert np.all(np.abs(got[..., 5] - ref[..., 5]) <= 1e-12 * (np.abs(ref[..., 5]) + 1e-6 * np.abs(ref[..., 5]).max())), name
        assert np.any(ref[..., 6:9] != 0.), name   # the rewritten components are not trivially zero
