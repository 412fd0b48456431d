"""Train the warm-start network of the implicit radiation solve on the GPU.

    python -m koral_b200.train_warmstart [--source cells|radtorus] [--n 16777216]
                                         [--epochs 24] [--out FILE]

Training pairs come from the product's own solver without a warm start,
solved to RADIMPCONV; the input is the cell's state before the solve (16
features), the target the change to the converged state (5 numbers); cells
whose solve fails are left out.  Two sources:
  cells     random radiating cells of the batched-solve distribution
            extended with a magnetic field (B^i g_ij B^j / rho log-uniform in
            [1e-3, 1e3]);
  radtorus  the cells of the radiative torus (256x128x64) as its own RK2IMEX
            run solves them, one implicit step per time step.  The network (16 -> 128 -> 128 -> 5, BF16 tensor-core kernels
with FP32 accumulation) is trained with Adam by the library's own forward
and backward kernels; the outputs are standardised with the targets' mean
and standard deviation, which are stored with the weights.  The velocity
outputs are standardised with three times their deviation, which weights
the two energy outputs nine times more in the loss: the Newton iteration
limits how far an energy may move per step (a factor of ten), so the
energies are what a warm start must get right.  Two more outputs score
whether the plain solve's first attempt, and its first two attempts,
failed (targets 1/0): the solver begins a warm-started cell with the first
energy-equation attempt expected to succeed.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "warmstart_mlp.npz")
DEFAULT_OUT_RADTORUS = os.path.join(HERE, "data", "warmstart_radtorus.npz")
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
        po, _, st, at, _, _ = k.rad_solve_device(rp, *d)
        X = k.rad_features_device(rp, d[1], d[2], d[3], d[4])
        T = k.rad_targets_device(rp, d[1], po, d[2], d[3], st, at)
        ok = torch.isfinite(T).all(dim=1) & torch.isfinite(X).all(dim=1)
        Xs.append(X[ok])
        Ts.append(T[ok])
        done += m
        c += 1
        log(f"  pairs {done}/{n}: kept {int(ok.sum())} of {m}")
    return torch.cat(Xs), torch.cat(Ts)


def make_pairs_radtorus(k, rp, n, log=print, shape=(256, 128, 64), skip=3):
    """Features and targets of the implicit solves of a radiative torus run
    (the second implicit step of each time step, after `skip` steps), and
    the running context."""
    import torch
    s = k.radtorus(*shape, rp=rp)
    s.set_implicit_solver(k.RAD_BATCHED, None)
    if skip:
        s.rk2imex_steps(skip, graph=True)
    Xs, Ts = [], []
    done = 0
    step = 0
    while done < n:
        s.rk2imex_steps(1, graph=True)
        X, T = s.implicit_pairs(rp)
        ok = torch.isfinite(T).all(dim=1) & torch.isfinite(X).all(dim=1)
        m = min(int(ok.sum()), n - done)
        Xs.append(X[ok][:m])
        Ts.append(T[ok][:m])
        done += m
        step += 1
        log(f"  torus step {step}: pairs {done}/{n}")
    return torch.cat(Xs), torch.cat(Ts), s


def evaluate_radtorus(k, mlp, rp, s, advance=2, warm_attempts=2, skip=2):
    """Held-out: the torus run advanced further, then one implicit step from
    the same state without and with the network (mean Newton iterations per
    solve over all attempts, failed solves, fallbacks), the network used as
    the radiative-torus benchmark uses it (warm starts for the first two
    attempts, only for cells the network expects to fail their first)."""
    s.set_implicit_solver(k.RAD_BATCHED, None)
    s.rk2imex_steps(advance, graph=True)
    u, p = s.download_state()
    dt = (1. - 2. ** -0.5) / s.tstepdenmax
    res = {"warm_attempts": warm_attempts, "skip": skip}
    s.set_implicit_options(warm_attempts=warm_attempts, skip=skip)
    for tag, warm in (("plain", None), ("learned", mlp)):
        s.set_implicit_solver(k.RAD_BATCHED, warm)
        s.upload_state(u.copy(), p.copy())
        s.reset_counters()
        s.op_implicit(0., dt)
        c = s.counters()
        res[tag] = dict(iterations=c["imp_iters"] / max(1, c["imp_solves"]), failed=int(c["radimp_failed"]),
                        fallbacks=int(c["imp_fallbacks"]), solves=int(c["imp_solves"]))
    res["ratio"] = res["plain"]["iterations"] / max(1e-300, res["learned"]["iterations"])
    return res


VELOCITY_WEIGHT = 3.0
SCORE_SCALE = 0.5


def evaluate(k, mlp, rp, n=1 << 16, seed=99001, sigma=SIGMA):
    """Plain against learned solve on held-out cells: mean Newton iterations
    per solve over all attempts and of the succeeding attempt, fallback
    rate, status agreement, median error of the predicted energies."""
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
    return dict(plain_iterations_all_attempts=plain[5][0] / n, learned_iterations_all_attempts=warm[5][0] / n,
                ratio_all_attempts=plain[5][0] / max(1, warm[5][0]),
                plain_iterations=float(ip[ok].mean()), learned_iterations=float(iw[ok].mean()),
                ratio=float(ip[ok].mean() / iw[ok].mean()), fallback_rate=warm[5][2] / n,
                status_agreement=float(np.mean(sp == sw)), guess_error_median_u=float(np.median(err[ok, 0])),
                guess_error_median_E=float(np.median(err[ok, 1])), cells=n, seed=seed)


def train(n=1 << 24, epochs=24, batch=8192, lr=2e-3, decay=0.85, seed=4000, out=None, log=print, source="cells"):
    import torch
    import koral_b200 as k
    t0 = time.time()
    if source == "radtorus":
        rp = k.rad_params(mass=k.RADTORUS_MASS, gamma=13.0 / 9.0)
        X, T, run = make_pairs_radtorus(k, rp, n, log=log)
        out = out or DEFAULT_OUT_RADTORUS
    else:
        rp = k.rad_params()
        X, T = make_pairs(k, rp, n, seed, log=log)
        out = out or DEFAULT_OUT
    t1 = time.time()
    mlp = k.Mlp(seed=7)
    blob = mlp.get()
    nout = k.MLP_OUT
    mean = T.mean(0).cpu().numpy()
    std = T.std(0).cpu().numpy()
    size = blob.size
    scale = np.maximum(std, 1e-6)
    scale[2:5] *= VELOCITY_WEIGHT
    # the attempt scores: raw 0/1 outputs (mean 0), weighted in the loss as
    # a unit-variance output (scale 0.5)
    mean[5:7] = 0.
    scale[5:7] = SCORE_SCALE
    blob[size - 16:size - 16 + nout] = mean
    blob[size - 8:size - 8 + nout] = scale
    mlp.set(blob)
    losses = []
    for e in range(epochs):
        rate = lr * (decay ** e)
        losses.append(mlp.train_epoch(X, T, batch=batch, lr=rate, seed=seed + e))
        log(f"  epoch {e}: lr {rate:.2e} mean loss {losses[-1]:.5f}")
    torch.cuda.synchronize()
    t2 = time.time()
    meta = dict(source=source, pairs=int(X.shape[0]), cells=n, epochs=epochs, batch=batch, lr=lr, decay=decay,
                seed=seed, losses=losses, pair_seconds=t1 - t0, train_seconds=t2 - t1)
    if source == "radtorus":
        meta["held_out"] = evaluate_radtorus(k, mlp, rp, run)
    else:
        meta["sigma"] = list(SIGMA)
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
    ap.add_argument("--out", default=None)
    ap.add_argument("--source", default="cells", choices=["cells", "radtorus"])
    a = ap.parse_args()
    sys.path.insert(0, os.path.dirname(HERE))
    train(a.n, a.epochs, a.batch, a.lr, a.decay, out=a.out, log=lambda s: print(s, flush=True), source=a.source)


if __name__ == "__main__":
    main()
