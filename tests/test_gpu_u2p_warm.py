"""The MHD inversion on device cells (kgpu_u2p_cells_device) and its learned
warm start.

Cells: random radiating cells with a magnetic field (B^2/rho log-uniform in
[1e-3, 1e3]); the gas part of each cell's conserved state after the plain
implicit solve is inverted from the primitives before the solve.

* Without a prediction the entry point is the reference's u2p: against the
  reference build's own u2p (u2p.c:176) the statuses are equal and the MHD
  primitives bit-identical except the entropy, which goes through CUDA's
  log and pow (1e-12 relative).
* A prediction gated off everywhere (wgate above every output, sgate above
  every score) takes the reference's path: the same bits and iteration
  counts as no prediction.
* The trained network (koral_b200/data/warmstart_u2p.npz) with the default
  gates takes no more Newton iterations over all solves than the plain
  inversion, needs the fallback in at most 1% of cells and agrees on the
  status in 99.9%.  Where both used the energy equation, the density and W
  differ from the plain inversion's by no more than ten times the plain
  inversion's own spread when its guess is moved by 0.1% (the size of the
  network's error): both are Newton iterations on the same equation to
  U2PCONV = 1e-10, whose stopping test (a relative step or a relative
  residual below 1e-10) leaves ill-conditioned cells that far apart.
"""
import os

import numpy as np
import pytest

from conftest import ref_lib_available

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(os.path.dirname(HERE), "koral_b200", "data", "warmstart_u2p.npz")


@pytest.fixture(scope="module")
def cells(kgpu):
    from koral_b200 import train_warmstart as tw
    rp = kgpu.rad_params()
    U, P0, g, G = tw.u2p_cells(kgpu, rp, 1 << 14, 31337)
    return rp, kgpu.u2p_config(rp.gamma), U, P0, g, G


@pytest.mark.skipif(not ref_lib_available("libkref_radcells.so"), reason="reference radiating-cells build not present")
def test_plain_device_inversion_matches_reference(kgpu, oracle, cells):
    rp, cfg, U, P0, g, G = cells
    n = 4096
    uu, pp, gh, Gh = (a[:n].cpu().numpy() for a in (U, P0, g, G))
    ref = oracle.RefRadCells()
    pr, sr, _, _ = ref.u2p_full(uu, pp, gh, Gh)
    pd, sd, fd, it, stats = kgpu.u2p_cells_device(cfg, U[:n], P0[:n], g[:n], G[:n])
    pd, sd = pd.cpu().numpy(), sd.cpu().numpy()
    assert np.array_equal(sd, sr)
    print("statuses", np.unique(sr, return_counts=True), "iterations per inversion", stats[0] / n)
    mhd = [0, 1, 2, 3, 4, 6, 7, 8]
    assert np.array_equal(pd[:, mhd], pr[:, mhd])
    rel = np.abs(pd[:, 5] - pr[:, 5]) / (np.abs(pr[:, 5]) + 1e-300)
    assert rel.max() <= 1e-12, rel.max()
    # and the host-pointer entry point gives the same bits
    ph, sh, fh = kgpu.u2p_cells(cfg, uu[:, :9], pp[:, :9], gh, Gh)
    assert np.array_equal(ph, pd[:, :9]) and np.array_equal(sh, sd) and np.array_equal(fh, fd.cpu().numpy())
    assert stats[0] == int(it.sum().item())


def test_gated_off_prediction_is_the_reference_path(kgpu, torch, cells):
    rp, cfg, U, P0, g, G = cells
    n = U.shape[0]
    Y = torch.full((n, 8), 0.3, dtype=torch.float32, device=U.device)
    Y[:, 1] = 0.9
    a = kgpu.u2p_cells_device(cfg, U, P0, g, G)
    b = kgpu.u2p_cells_device(cfg, U, P0, g, G, ypred=Y, wgate=1.0, sgate=1.0)
    for x, y in zip(a[:4], b[:4]):
        assert torch.equal(x, y)
    assert a[4][0] == b[4][0] and b[4][1] == 0


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained u2p warm-start weights")
def test_trained_u2p_warm_start(kgpu, torch, cells):
    from koral_b200 import train_warmstart as tw
    rp, cfg, U, P0, g, G = cells
    n = U.shape[0]
    mlp = tw.load(kgpu, WEIGHTS)
    X = kgpu.u2p_features_device(cfg, U, P0, g, G)
    Y = mlp.forward(X)
    plain = kgpu.u2p_cells_device(cfg, U, P0, g, G)
    warm = kgpu.u2p_cells_device(cfg, U, P0, g, G, ypred=Y)
    sp, sw = plain[1].cpu().numpy(), warm[1].cpu().numpy()
    print(f"iterations per inversion: plain {plain[4][0] / n:.4f}, learned {warm[4][0] / n:.4f}; "
          f"fallbacks {warm[4][1]}, status agreement {np.mean(sp == sw):.6f}")
    assert warm[4][0] <= plain[4][0]
    assert warm[4][1] <= 0.01 * n
    assert np.mean(sp == sw) >= 0.999
    Pn = P0.clone()
    Pn[:, 0] *= 1.001
    Pn[:, 1] *= 1.001
    nudged = kgpu.u2p_cells_device(cfg, U, Pn, g, G)
    sn = nudged[1].cpu().numpy()
    gamma = rp.gamma
    gg = g.cpu().numpy().reshape(-1, 4, 5)[:, 1:4, 1:4]

    def wof(p):
        v = p[:, 2:5]
        return (p[:, 0] + gamma * p[:, 1]) * (1 + np.einsum("ni,nij,nj->n", v, gg, v))

    def spread(a, b, mask):
        a, b = a[0].cpu().numpy(), b[0].cpu().numpy()
        rho = np.abs(a[:, 0] - b[:, 0]) / a[:, 0]
        w = np.abs(wof(a) - wof(b)) / wof(a)
        return rho[mask], w[mask]
    rho_l, w_l = spread(plain, warm, (sp == 0) & (sw == 0))
    rho_n, w_n = spread(plain, nudged, (sp == 0) & (sn == 0))
    print(f"largest relative difference from the plain inversion: learned start density {rho_l.max():.3e} "
          f"W {w_l.max():.3e}; guess moved by 0.1%: density {rho_n.max():.3e} W {w_n.max():.3e}")
    assert rho_l.max() <= max(10 * rho_n.max(), 1e-14) and w_l.max() <= max(10 * w_n.max(), 1e-14)
