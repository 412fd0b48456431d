"""kgpu_u2p_cells_static (batched u2p from a static device array, no
allocation) against kgpu_u2p_cells on the same cells, two calls in a row.

The cells sit at metric points of the MKS2 Kerr grid (spin 0.9) built by the
library's own host-side metric code, so nothing outside the repository is
needed.  Tolerance: none.  Both entry points run the same inversion code
built with the same flags, so status, fixup flags and all nine primitives
(entropy included) must be bit-identical.  The second call has a different
batch size and different cells, so stale contents of the shared array from
the first call would show up.  A third call is bracketed by the device's
free-memory figure, which must not move: the entry point allocates nothing.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def kerr_points(kgpu):
    tp = kgpu.torus_params()
    cfg = kgpu.torus_config(24, 16, 8)
    ng = cfg.ng
    xb = [np.log(tp.r_lo) + (np.log(tp.r_hi) - np.log(tp.r_lo)) * (np.arange(-ng, cfg.nx + ng + 1) / cfg.nx),
          tp.x2_lo + (tp.x2_hi - tp.x2_lo) * (np.arange(-ng, cfg.ny + ng + 1) / cfg.ny),
          2 * np.pi * np.arange(-ng, cfg.nz + ng + 1) / cfg.nz]
    g, G = kgpu.mks2_metric_tables(tp, cfg, xb)[:2]
    g, G = g.reshape(-1, 20), G.reshape(-1, 20)
    ok = np.isfinite(g).all(axis=1) & np.isfinite(G).all(axis=1) & (g[:, 19] > 0)
    return cfg, g[ok], G[ok]


def cells(cfg, g, G, n, seed, kgpu):
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, len(g), n)
    gm, Gm = g[idx].copy(), G[idx].copy()
    pp = np.zeros((n, 9))
    pp[:, 0] = 10 ** rng.uniform(-5, 0, n)
    pp[:, 1] = pp[:, 0] * 10 ** rng.uniform(-4, 1, n)
    pp[:, 2:5] = rng.normal(0, 0.5, (n, 3))
    pp[:, 6:9] = rng.normal(0, 0.1, (n, 3)) * np.sqrt(pp[:, :1])
    gam = cfg.gamma
    pp[:, 5] = pp[:, 0] * np.log(((gam - 1) * pp[:, 1]) ** (1 / (gam - 1)) / pp[:, 0] ** (1 / (gam - 1) + 1))
    uu = kgpu.p2u_cells(cfg, pp, gm, Gm)
    guess = pp * (1 + rng.uniform(-0.05, 0.05, pp.shape))
    return uu, guess, gm, Gm


def test_static_u2p_matches_allocating_entry_point(kgpu):
    cfg, g, G = kerr_points(kgpu)
    assert len(g) > 100
    for call, (n, seed) in enumerate([(kgpu.STATIC_MAX_CELLS, 11), (3001, 12)]):
        uu, guess, gm, Gm = cells(cfg, g, G, n, seed, kgpu)
        pa, sa, fa = kgpu.u2p_cells(cfg, uu, guess, gm, Gm)
        ps, ss, fs = kgpu.u2p_cells_static(cfg, uu, guess, gm, Gm)
        assert np.array_equal(ss, sa), f"call {call}: status differs"
        assert np.array_equal(fs, fa), f"call {call}: fixup flags differ"
        assert (sa == 0).mean() > 0.9
        assert np.array_equal(ps, pa), f"call {call}: primitives differ"


def test_static_u2p_allocates_nothing(kgpu):
    """Free device memory before and after a call of the static entry point
    (after a first call, which may load the library's module and with it
    the static array) is the same to the byte."""
    import torch
    cfg, g, G = kerr_points(kgpu)
    uu, guess, gm, Gm = cells(cfg, g, G, 2048, 13, kgpu)
    kgpu.u2p_cells_static(cfg, uu, guess, gm, Gm)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    ps, ss, fs = kgpu.u2p_cells_static(cfg, uu, guess, gm, Gm)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    assert (ss == 0).mean() > 0.9


def test_static_u2p_rejects_oversize_batch(kgpu):
    cfg, g, G = kerr_points(kgpu)
    n = kgpu.STATIC_MAX_CELLS + 1
    uu = np.zeros((n, 9))
    with pytest.raises(kgpu.KgpuError, match="static limit"):
        kgpu.u2p_cells_static(cfg, uu, uu, np.zeros((n, 20)), np.zeros((n, 20)))
    header = open(os.path.join(os.path.dirname(__file__), "..", "include", "koral_b200.h")).read()
    assert f"#define KGPU_STATIC_MAX_CELLS {kgpu.STATIC_MAX_CELLS}" in header
