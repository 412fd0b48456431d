"""The warm-start network's tensor-core kernels against the numpy oracle
(oracle/mlp_oracle.py), and the warm start's plumbing in the batched
implicit solve.

Tolerances: the device evaluates SiLU with the fast exponential and rounds
activations to BF16, the oracle with numpy's exponential and the same
rounding; a last-place difference before a rounding can move one BF16
activation by one unit (2^-8 relative), so outputs agree to 2e-2 absolute
(they are O(1)) and gradients to 2% in norm with a cosine above 0.999.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def _random_setup(kgpu, n, seed):
    rng = np.random.default_rng(seed)
    m = kgpu.Mlp(seed=seed)
    blob = m.get()
    blob[-16:-9] = rng.normal(0, 0.1, 7)
    blob[-8:-1] = rng.uniform(0.5, 2.0, 7)
    m.set(blob)
    X = rng.normal(0, 1, (n, 16)).astype(np.float32)
    T = rng.normal(0, 1, (n, 7)).astype(np.float32)
    return m, m.get(), X, T


def test_mlp_forward_matches_oracle(kgpu, torch):
    from oracle import mlp_oracle as mo
    m, blob, X, _ = _random_setup(kgpu, 1000, 3)
    Y = m.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    ref = mo.predict(blob, X)
    d = np.abs(Y[:, :7] - ref[:, :7])
    print("forward: max abs diff", d.max(), "mean", d.mean())
    assert d.max() <= 2e-2 and d.mean() <= 1e-3


def test_mlp_gradient_matches_oracle(kgpu, torch):
    from oracle import mlp_oracle as mo
    m, blob, X, T = _random_setup(kgpu, 512, 4)
    g, loss = m.gradient(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    lref, gref = mo.gradient(blob, X, T)
    assert abs(loss - lref) <= 1e-3 * lref
    blocks = dict(W1=(mo.OW1, mo.OB1), b1=(mo.OB1, mo.OW2), W2=(mo.OW2, mo.OB2), b2=(mo.OB2, mo.OW3),
                  W3=(mo.OW3, mo.OB3), b3=(mo.OB3, mo.NPARAM))
    for name, (a, b) in blocks.items():
        x, y = g[a:b].astype(np.float64), gref[a:b]
        rel = np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30)
        cos = float(x @ y / max(np.linalg.norm(x) * np.linalg.norm(y), 1e-30))
        print(f"{name}: relative difference {rel:.2e}, cosine {cos:.6f}")
        assert rel <= 2e-2 and cos >= 0.999, name


def _solved_pairs(kgpu, torch, n, seed):
    rp = kgpu.rad_params()
    uu, pp, g, G, dt = kgpu.rad_cells(n, seed, rp, sigma=(1e-3, 1e3))
    d = [torch.from_numpy(a).cuda() for a in (uu, pp, g, G, dt)]
    po, _, st, at, _, _ = kgpu.rad_solve_device(rp, *d)
    X = kgpu.rad_features_device(rp, d[1], d[2], d[3], d[4])
    T = kgpu.rad_targets_device(rp, d[1], po, d[2], d[3], st, at)
    ok = torch.isfinite(T).all(dim=1) & torch.isfinite(X).all(dim=1)
    return rp, d, X, T, ok


def test_mlp_training_lowers_the_loss(kgpu, torch):
    rp, d, X, T, ok = _solved_pairs(kgpu, torch, 1 << 15, 11)
    X, T = X[ok].contiguous(), T[ok].contiguous()
    m = kgpu.Mlp(seed=5)
    blob = m.get()
    blob[-16:-9] = T.mean(0).cpu().numpy()
    blob[-8:-1] = T.std(0).cpu().numpy().clip(1e-3)
    m.set(blob)
    losses = [m.train_epoch(X, T, batch=1024, lr=2e-3, seed=e) for e in range(4)]
    print("losses", losses)
    assert losses[-1] < 0.7 * losses[0]


def test_warm_start_with_the_guess_itself_is_the_plain_solve(kgpu, torch):
    """A prediction of 'no change' makes the warm iterate the cell's own
    guess: every output equals the plain batched solve's, bit for bit, and
    the fallbacks (cells whose whole warm cascade fails, then rerun from the
    guess) are exactly the cells the plain solve cannot solve."""
    rp = kgpu.rad_params()
    uu, pp, g, G, dt = kgpu.rad_cells(8192, 21, rp)
    d = [torch.from_numpy(a).cuda() for a in (uu, pp, g, G, dt)]
    a = kgpu.rad_solve_device(rp, *d)
    zero = torch.zeros((8192, 8), dtype=torch.float32, device="cuda")
    b = kgpu.rad_solve_device(rp, *d, ypred=zero)
    for x, y in zip(a[:5], b[:5]):
        assert torch.equal(x, y)
    assert b[5][2] == int((a[2] != 0).sum())


WEIGHTS = os.path.join(os.path.dirname(__file__), "..", "koral_b200", "data", "warmstart_mlp.npz")


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained warm-start weights")
def test_trained_warm_start_cuts_newton_iterations(kgpu, torch):
    """The trained network on held-out cells (seed not used in training):
    Newton iterations per implicit solve counted over every attempt the
    solve makes (failed attempts, skipped ones not run, and the fallback to
    the reference cascade included) at least 2x fewer than the plain
    batched solve at the same residual, and the same success on 99% of the
    cells."""
    from koral_b200 import train_warmstart
    m = train_warmstart.load(kgpu, WEIGHTS)
    rp = kgpu.rad_params()
    uu, pp, g, G, dt = kgpu.rad_cells(1 << 16, 99001, rp, sigma=(1e-3, 1e3))
    d = [torch.from_numpy(a).cuda() for a in (uu, pp, g, G, dt)]
    plain = kgpu.rad_solve_device(rp, *d)
    X = kgpu.rad_features_device(rp, d[1], d[2], d[3], d[4])
    Y = m.forward(X)
    warm = kgpu.rad_solve_device(rp, *d, ypred=Y)
    ip, iw = plain[4].cpu().numpy(), warm[4].cpu().numpy()
    sp, sw = plain[2].cpu().numpy(), warm[2].cpu().numpy()
    ok = (sp == 0) & (sw == 0)
    all_plain, all_warm = plain[5][0] / len(sp), warm[5][0] / len(sp)
    print(f"iterations per solve over all attempts: plain {all_plain:.3f} learned {all_warm:.3f} "
          f"(ratio {all_plain / all_warm:.3f}); succeeding attempt: plain {ip[ok].mean():.3f} "
          f"learned {iw[ok].mean():.3f}; fallbacks {warm[5][2]}; status agree {np.mean(sp == sw):.4f}")
    assert np.mean(sp == sw) >= 0.99
    assert all_warm * 2.0 <= all_plain
