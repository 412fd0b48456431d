"""Train the warm-start network of the implicit radiation solve on the GPU.

    python -m koral_b200.train_warmstart [--n 16777216] [--epochs 6] [--out FILE]

Training pairs come from the product's own plain solver: random radiating
cells of the batched-solve distribution extended with a magnetic field
(B^i g_ij B^j / rho log-uniform in [1e-3, 1e3]), solved to RADIMPCONV; the
input is the cell's state before the solve (16 features), the target the
change to the converged state (5 numbers).  Cells whose solve fails are
left out.  The network (16 -> 128 -> 128 -> 5, BF16 tensor-core kernels
with FP32 accumulation) is trained with Adam by the library's own forward
and backward kernels; the outputs are standardised with the targets' mean
and standard deviation, which are stored with the weights.  The velocity
outputs are standardised with three times their deviation, which weights
the two energy outputs nine times more in the loss: the Newton iteration
limits how far an energy may move per step (a factor of ten), so the
energies are what a warm start must get right.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "warmstart_mlp.npz")
SIGMA = (1e-3, 1e3)


def make_pairs(k, rp, n, seed, chunk=1 << 20, log=print):
    """Features and targets (device tensors) of n solved cells."""
    import torch
    Xs, Ts = [], []
    done = 0
    c = 0
    while done < n:
        m = min(chunk, n - done)
        uu, pp, g, G, dt = k.rad_cells(m, seed + c, rp, sigma=SIGMA)
        d = [torch.from_numpy(a).cuda() for a in (uu, pp, g, G, dt)]
        po, _, st, _, _, _ = k.rad_solve_device(rp, *d)
        X = k.rad_features_device(rp, d[1], d[2], d[3], d[4])
        T = k.rad_targets_device(rp, d[1], po, d[2], d[3], st)
        ok = torch.isfinite(T).all(dim=1) & torch.isfinite(X).all(dim=1)
        Xs.append(X[ok])
        Ts.append(T[ok])
        done += m
        c += 1
        log(f"  pairs {done}/{n}: kept {int(ok.sum())} of {m}")
    return torch.cat(Xs), torch.cat(Ts)


VELOCITY_WEIGHT = 3.0


def evaluate(k, mlp, rp, n=1 << 16, seed=99001, sigma=SIGMA):
    """Plain against learned solve on held-out cells: mean Newton iterations
    of the succeeding attempt, fallback rate, status agreement, median error
    of the predicted energies."""
    import torch
    uu, pp, g, G, dt = k.rad_cells(n, seed, rp, sigma=sigma)
    d = [torch.from_numpy(a).cuda() for a in (uu, pp, g, G, dt)]
    plain = k.rad_solve_device(rp, *d)
    X = k.rad_features_device(rp, d[1], d[2], d[3], d[4])
    Y = mlp.forward(X)
    warm = k.rad_solve_device(rp, *d, ypred=Y)
    sp, sw = plain[2].cpu().numpy(), warm[2].cpu().numpy()
    ip, iw = plain[4].cpu().numpy(), warm[4].cpu().numpy()
    ok = (sp == 0) & (sw == 0)
    true = (plain[0][:, [1, 9]] / d[1][:, [1, 9]]).cpu().numpy()
    pred = np.exp(Y[:, :2].double().cpu().numpy())
    err = np.abs(pred - true) / np.abs(true)
    return dict(plain_iterations=float(ip[ok].mean()), learned_iterations=float(iw[ok].mean()),
                ratio=float(ip[ok].mean() / iw[ok].mean()), fallback_rate=warm[5][2] / n,
                status_agreement=float(np.mean(sp == sw)), guess_error_median_u=float(np.median(err[ok, 0])),
                guess_error_median_E=float(np.median(err[ok, 1])), cells=n, seed=seed)


def train(n=1 << 24, epochs=24, batch=8192, lr=2e-3, decay=0.85, seed=4000, out=DEFAULT_OUT, log=print):
    import torch
    import koral_b200 as k
    rp = k.rad_params()
    t0 = time.time()
    X, T = make_pairs(k, rp, n, seed, log=log)
    t1 = time.time()
    mlp = k.Mlp(seed=7)
    blob = mlp.get()
    mean = T.mean(0).cpu().numpy()
    std = T.std(0).cpu().numpy()
    size = blob.size
    blob[size - 16:size - 16 + 5] = mean
    scale = np.maximum(std, 1e-6)
    scale[2:5] *= VELOCITY_WEIGHT
    blob[size - 8:size - 8 + 5] = scale
    mlp.set(blob)
    losses = []
    for e in range(epochs):
        rate = lr * (decay ** e)
        losses.append(mlp.train_epoch(X, T, batch=batch, lr=rate, seed=seed + e))
        log(f"  epoch {e}: lr {rate:.2e} mean loss {losses[-1]:.5f}")
    torch.cuda.synchronize()
    t2 = time.time()
    meta = dict(pairs=int(X.shape[0]), cells=n, epochs=epochs, batch=batch, lr=lr, decay=decay, seed=seed,
                losses=losses, pair_seconds=t1 - t0, train_seconds=t2 - t1, sigma=list(SIGMA))
    meta["held_out"] = evaluate(k, mlp, rp)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    np.savez(out, blob=mlp.get(), meta=json.dumps(meta))
    log(json.dumps(meta))
    return mlp, meta


def load(k, path=DEFAULT_OUT):
    """A network with the stored weights."""
    d = np.load(path)
    m = k.Mlp(seed=1)
    m.set(d["blob"])
    return m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 24)
    ap.add_argument("--epochs", type=int, default=24)
    ap.add_argument("--decay", type=float, default=0.85)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    sys.path.insert(0, os.path.dirname(HERE))
    train(a.n, a.epochs, a.batch, a.lr, a.decay, out=a.out, log=lambda s: print(s, flush=True))


if __name__ == "__main__":
    main()
