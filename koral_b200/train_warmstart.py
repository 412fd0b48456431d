"""Train the warm-start network of the implicit radiation solve on the GPU.

    python -m koral_b200.train_warmstart [--source cells|radtorus|u2p] [--n 16777216]
                                         [--epochs 24] [--out FILE]

Training pairs come from the product's own solver without a warm start,
solved to RADIMPCONV; the input is the cell's state before the solve (16
features), the target the change to the converged state (5 numbers); cells
whose solve fails are left out.  Sources:
  cells     random radiating cells of the batched-solve distribution
            extended with a magnetic field (B^i g_ij B^j / rho log-uniform in
            [1e-3, 1e3]);
  radtorus  the cells of the radiative torus (256x128x64) as its own RK2IMEX
            run solves them, one implicit step per time step;
  u2p       the warm start of the MHD inversion instead: the gas part of the
            conserved state after the plain implicit solve of the cells
            above, inverted by the reference's u2p from the primitives
            before it; targets ln(W / W_guess) and whether the entropy
            equation was needed.
The network (16 -> 128 -> 128 -> 5, BF16 tensor-core kernels
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
DEFAULT_OUT_U2P = os.path.join(HERE, "data", "warmstart_u2p.npz")
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


def u2p_cells(k, rp, n, seed, sigma=SIGMA):
    """Inversion problems of the batched-solve distribution with a magnetic
    field: the gas part of each cell's conserved state after the plain
    implicit solve, to be inverted from the primitives before it (the
    situation of calc_u2p after a step that moved the gas energy by the
    radiation exchange).  Cells whose solve failed are left out.  Returns
    device tensors (uu, pp_guess, g, G)."""
    import torch
    uu, pp, g, G, dt = k.rad_cells(n, seed, rp, sigma=sigma)
    d = [torch.from_numpy(a).cuda() for a in (uu, pp, g, G, dt)]
    po, uo, st, at, _, _ = k.rad_solve_device(rp, *d)
    ok = st == 0
    return uo[ok].contiguous(), d[1][ok].contiguous(), d[2][ok].contiguous(), d[3][ok].contiguous()


def subdomain_inversion_cells(k, s):
    """Inversion problems of a running subdomain, as calc_u2p meets them
    (finite.c:502): the conserved state after one explicit operator at the
    current time step, to be inverted from the primitives before it; domain
    cells only, with their centre metric.  The subdomain's state is put
    back.  Returns device tensors (uu, pp_guess, g, G)."""
    import torch
    u0, p0 = s.download_state()
    td = s.tstepdenmax
    dt = s.begin_step()
    s.op_explicit(0., dt)
    u1, _ = s.download_state()
    s.upload_state(u0, p0)
    s.tstepdenmax = td
    cfg = s.cfg
    ng = cfg.ng
    sl = tuple(slice(ng, -ng) if n > 1 else slice(None) for n in (cfg.nz, cfg.ny, cfg.nx))
    nv = cfg.nv
    U = u1[sl].reshape(-1, nv)
    P = p0[sl].reshape(-1, nv)
    g, G = s.download_metric()[:2]
    sx, sy = cfg.nx + 2 * ng, cfg.ny + 2 * ng
    szm = 1 if cfg.axisym_metric else (cfg.nz + 2 * ng if cfg.nz > 1 else 1)
    g = g.reshape(szm, sy, sx, 20)
    G = G.reshape(szm, sy, sx, 20)
    if cfg.axisym_metric:
        g = np.broadcast_to(g, (cfg.nz + 2 * ng if cfg.nz > 1 else 1, sy, sx, 20))
        G = np.broadcast_to(G, g.shape)
    gc = np.ascontiguousarray(g[sl].reshape(-1, 20))
    Gc = np.ascontiguousarray(G[sl].reshape(-1, 20))
    return tuple(torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (U, P, gc, Gc))


def inversion_stats(k, cfg, U, P0, g, G, mlp=None, wgate=None, sgate=None):
    """Newton iterations per inversion (all solves), where they go, and the
    learned warm start's figures when a network is given."""
    import torch
    plain = k.u2p_cells_device(cfg, U, P0, g, G)
    n = U.shape[0]
    st, it = plain[1].cpu().numpy(), plain[3].cpu().numpy()
    res = dict(cells=n, plain_iterations=plain[4][0] / n, plain_w_evaluations=plain[4][2] / n,
               entropy_rate=float(np.mean(st == -1)), failed_rate=float(np.mean(st < -1)),
               iterations_in_entropy_cells=float(it[st == -1].sum() / max(1, it.sum())),
               iteration_histogram=np.bincount(np.minimum(it, 60), minlength=61).tolist())
    if mlp is not None:
        X = k.u2p_features_device(cfg, U, P0, g, G)
        Y = mlp.forward(X)
        kw = {}
        if wgate is not None:
            kw["wgate"] = wgate
        if sgate is not None:
            kw["sgate"] = sgate
        warm = k.u2p_cells_device(cfg, U, P0, g, G, ypred=Y, **kw)
        sw = warm[1].cpu().numpy()
        res.update(learned_iterations=warm[4][0] / n, ratio=plain[4][0] / max(1, warm[4][0]),
                   learned_w_evaluations=warm[4][2] / n, fallback_rate=warm[4][1] / n,
                   status_agreement=float(np.mean(st == sw)))
    torch.cuda.synchronize()
    return res


def make_pairs_u2p(k, rp, n, seed, chunk=1 << 20, log=print):
    """Features and targets (device tensors) of n inversions solved by the
    reference's u2p from the guess (u2p_cells), half of them of cells with a
    magnetic field and half without."""
    import torch
    cfg = k.u2p_config(rp.gamma)
    Xs, Ts = [], []
    done = 0
    c = 0
    while done < n:
        # alternate chunks with and without a magnetic field
        U, P0, g, G = u2p_cells(k, rp, min(chunk, n - done), seed + c, sigma=SIGMA if c % 2 == 0 else None)
        P1, s1, _, _, _ = k.u2p_cells_device(cfg, U, P0, g, G)
        X = k.u2p_features_device(cfg, U, P0, g, G)
        T = k.u2p_targets_device(cfg, P0, P1, g, G, s1)
        ok = torch.isfinite(T).all(dim=1) & torch.isfinite(X).all(dim=1)
        m = min(int(ok.sum()), n - done)
        Xs.append(X[ok][:m])
        Ts.append(T[ok][:m])
        done += m
        c += 1
        log(f"  u2p pairs {done}/{n}")
    return torch.cat(Xs), torch.cat(Ts)


def evaluate_u2p(k, mlp, rp, n=1 << 16, seed=99001, sigma=SIGMA):
    """Plain against learned inversion on held-out cells: Newton iterations
    per inversion over all its solves, W-function evaluations, fallback
    rate, status agreement, the largest relative difference of the
    primitives where both succeed, median error of the predicted W, and
    device time of each (the learned time includes features and network)."""
    import torch
    cfg = k.u2p_config(rp.gamma)
    U, P0, g, G = u2p_cells(k, rp, n, seed, sigma=sigma)
    m = U.shape[0]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    k.u2p_cells_device(cfg, U, P0, g, G)   # warm-up
    torch.cuda.synchronize()
    ev[0].record()
    plain = k.u2p_cells_device(cfg, U, P0, g, G)
    ev[1].record()
    X = k.u2p_features_device(cfg, U, P0, g, G)
    Y = mlp.forward(X)
    warm = k.u2p_cells_device(cfg, U, P0, g, G, ypred=Y)
    ev[2].record()
    torch.cuda.synchronize()
    sp, sw = plain[1].cpu().numpy(), warm[1].cpu().numpy()
    both = (sp >= -1) & (sw >= -1)
    a, b = plain[0][:, :5].cpu().numpy(), warm[0][:, :5].cpu().numpy()
    rel = np.abs(a - b) / np.maximum(np.abs(a), 1e-300)
    T = k.u2p_targets_device(cfg, P0, plain[0], g, G, plain[1])
    ok = (sp >= -1) & np.isfinite(T[:, 0].cpu().numpy())
    werr = np.abs(np.expm1(Y[:, 0].double().cpu().numpy() - T[:, 0].double().cpu().numpy()))
    ms_plain, ms_warm = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    return dict(cells=m, seed=seed, plain_iterations=plain[4][0] / m, learned_iterations=warm[4][0] / m,
                ratio=plain[4][0] / max(1, warm[4][0]), plain_w_evaluations=plain[4][2] / m,
                learned_w_evaluations=warm[4][2] / m, fallback_rate=warm[4][1] / m,
                plain_entropy_rate=float(np.mean(sp == -1)), status_agreement=float(np.mean(sp == sw)),
                primitives_max_rel_diff_median=float(np.median(rel[both].max(axis=1))) if both.any() else None,
                w_error_median=float(np.median(werr[ok])) if ok.any() else None,
                plain_ms=ms_plain, learned_ms=ms_warm, plain_inversions_per_s=m / (ms_plain / 1e3),
                learned_inversions_per_s=m / (ms_warm / 1e3))


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
    elif source == "u2p":
        rp = k.rad_params()
        X, T = make_pairs_u2p(k, rp, n, seed, log=log)
        out = out or DEFAULT_OUT_U2P
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
    if source == "u2p":
        # one regression output and one score; the unused outputs are
        # zero targets with unit scale
        mean[1:] = 0.
        scale[1] = SCORE_SCALE
        scale[2:] = 1.
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
    elif source == "u2p":
        meta["sigma"] = list(SIGMA)
        meta["held_out"] = evaluate_u2p(k, mlp, rp)
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
    ap.add_argument("--source", default="cells", choices=["cells", "radtorus", "u2p"])
    a = ap.parse_args()
    sys.path.insert(0, os.path.dirname(HERE))
    train(a.n, a.epochs, a.batch, a.lr, a.decay, out=a.out, log=lambda s: print(s, flush=True), source=a.source)


if __name__ == "__main__":
    main()
