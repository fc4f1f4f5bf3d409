"""Train the warm-start network on converged reconstructions that the plain
method produces on seeded synthetic problems.

    python -m gpair_b200.train_warmstart --n64 16000 --n128 4000 --out gpair_b200/data/warmstart_cnn.npz

1. Problems (CPU, a spawn pool): seeded scenes of 1-10 Gaussians / disks /
   points (unit flux), random 4-12 telescope arrays, noise; 64x64 at 0.1 mas
   and 128x128 at 0.05 mas (gpair_b200.warmstart.training_case).
2. Targets (GPU): features (dirty images, uv density) and a CG reconstruction
   from the flat prior with the batched line search, `--iters` iterations;
   the target is the final image scaled to unit flux. Several contexts run
   concurrently, one per host thread, each on its own stream.
3. Training (GPU, the library's CUDA kernels): Adam, cosine learning rate,
   mini-batches of one image size; a share of the problems is held back for
   validation, which picks the learning rate when several are given.
Seeds of training problems are 0 .. n-1 (64^2) and 1e6 .. 1e6+n-1 (128^2);
held-out evaluation seeds start at 1e7.
"""
from __future__ import annotations

import argparse
import math
import os
import sys
import threading
import time
from typing import List, Sequence

import numpy as np

SEED_128 = 1_000_000
SEED_HELD_OUT = 10_000_000


def _case(args):
    seed, width = args
    from gpair_b200.warmstart import training_case
    return training_case(seed, width).problem


def make_problems(seeds_widths: Sequence, workers: int):
    import multiprocessing as mp
    if workers <= 1:
        return [_case(a) for a in seeds_widths]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_case, seeds_widths, chunksize=16)


def make_targets(problems: List, iters: int, threads: int, device: int = 0, log=print):
    """features [n, N_FEATURES, N, N] and unit-flux targets [n, N*N] for problems of one width."""
    import gpair_b200 as g
    from gpair_b200.warmstart import N_FEATURES, features
    n = len(problems)
    N = problems[0].width
    X = np.zeros((n, N_FEATURES, N, N), np.float32)
    T = np.zeros((n, N * N), np.float32)
    J = np.zeros(n, np.float64)
    nxt = [0]
    lock = threading.Lock()
    err: List[BaseException] = []

    def work():
        try:
            with g.Reconstructor(device) as rec:
                rec.set_precision(g.PREC_SPLIT16)
                while True:
                    with lock:
                        i = nxt[0]
                        nxt[0] += 1
                    if i >= n or err:
                        return
                    p = problems[i]
                    rec.set_problem(p)
                    X[i] = features(rec, p)
                    rec.set_image(p.start_image())
                    out = rec.cg(iters, method=2, line_search=g.LS_BATCH)
                    img = rec.get_image().astype(np.float64)
                    T[i] = (img / img.sum()).astype(np.float32)
                    J[i] = out["J"]
        except BaseException as e:  # noqa: BLE001
            err.append(e)

    t0 = time.time()
    ths = [threading.Thread(target=work) for _ in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    if err:
        raise err[0]
    log(f"targets: {n} problems of {N}x{N}, {iters} iterations each, {time.time() - t0:.1f} s")
    return X, T, J


def train(net, sets, epochs: int, batch: int, lr: float, log=print, seed: int = 0):
    """sets: list of (X, T) device tensors, one per image size. Returns per-epoch mean losses."""
    import torch
    rng = np.random.default_rng(seed)
    batches = []
    for si, (X, T) in enumerate(sets):
        n = X.shape[0]
        batches += [(si, k) for k in range(0, n - batch + 1, batch)] or [(si, 0)]
    total = epochs * len(batches)
    step, hist = 0, []
    for ep in range(epochs):
        perms = [torch.from_numpy(rng.permutation(X.shape[0])).to(X.device) for X, _ in sets]
        order = rng.permutation(len(batches))
        acc, cnt = 0.0, 0
        t0 = time.time()
        for bi in order:
            si, k = batches[bi]
            X, T = sets[si]
            idx = perms[si][k:k + batch]
            cur = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(total, 1)))
            loss = net.train_step(X[idx], T[idx], cur)
            acc += float(loss.sum())
            cnt += int(idx.numel())
            step += 1
        hist.append(acc / max(cnt, 1))
        log(f"epoch {ep + 1}/{epochs}: loss {hist[-1]:.5f} ({time.time() - t0:.1f} s)")
    return hist


def validate(net, sets, batch: int = 64) -> float:
    """Mean per-image loss over held-back (X, T) device tensors."""
    tot, cnt = 0.0, 0
    for X, T in sets:
        for k in range(0, X.shape[0], batch):
            out = net.forward(X[k:k + batch])
            loss, _ = net.loss_and_grad(out.reshape(out.shape[0], -1), T[k:k + batch], want_grad=False)
            tot += float(loss.sum())
            cnt += out.shape[0]
    return tot / max(cnt, 1)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n64", type=int, default=16000)
    ap.add_argument("--n128", type=int, default=4000)
    ap.add_argument("--iters", type=int, default=500, help="CG iterations of the target reconstructions")
    ap.add_argument("--epochs", type=int, default=16)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lrs", default=None, help="comma-separated learning rates; the best validation loss wins")
    ap.add_argument("--val-frac", type=float, default=0.05, help="problems held back for validation")
    ap.add_argument("--loss", choices=["relative", "absolute"], default="relative")
    ap.add_argument("--threads", type=int, default=8, help="concurrent CG contexts")
    ap.add_argument("--workers", type=int, default=0, help="CPU processes for problem generation (0: up to 32)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from gpair_b200.warmstart import DEFAULT_WEIGHTS, LOSS_ABSOLUTE, LOSS_RELATIVE, WarmStartNet
    workers = args.workers or min(32, os.cpu_count() or 1)
    log = lambda s: print(s, flush=True)  # noqa: E731
    t0 = time.time()
    specs = [(s, 64) for s in range(args.n64)] + [(SEED_128 + s, 128) for s in range(args.n128)]
    probs = make_problems(specs, workers)
    log(f"problems: {len(probs)} in {time.time() - t0:.1f} s on {workers} processes")
    sets_np = []
    for w in (64, 128):
        ps = [p for p in probs if p.width == w]
        if ps:
            X, T, _ = make_targets(ps, args.iters, args.threads, log=log)
            sets_np.append((X, T))
    import torch
    sets, vsets = [], []
    for X, T in sets_np:
        nv = int(round(args.val_frac * X.shape[0]))
        nt = X.shape[0] - nv
        sets.append((torch.from_numpy(X[:nt]).cuda(), torch.from_numpy(T[:nt]).cuda()))
        if nv:
            vsets.append((torch.from_numpy(X[nt:]).cuda(), torch.from_numpy(T[nt:]).cuda()))
    lrs = [float(v) for v in args.lrs.split(",")] if args.lrs else [args.lr]
    mode = LOSS_RELATIVE if args.loss == "relative" else LOSS_ABSOLUTE
    best = None
    for lr in lrs:
        net = WarmStartNet(None, 0, seed=0)
        net.loss_mode = mode
        t0 = time.time()
        hist = train(net, sets, args.epochs, args.batch, lr, log=log)
        v = validate(net, vsets) if vsets else hist[-1]
        log(f"lr {lr:g}: training {time.time() - t0:.1f} s, validation loss {v:.5f}")
        if best is None or v < best[0]:
            best = (v, lr, net, hist)
    v, lr, net, hist = best
    out = args.out or DEFAULT_WEIGHTS
    net.save(out, {"loss_history": np.asarray(hist), "n64": args.n64, "n128": args.n128, "iters": args.iters,
                   "epochs": args.epochs, "lr": lr, "val_loss": v, "loss_mode": mode})
    log(f"saved {out} (lr {lr:g}, validation loss {v:.5f})")


if __name__ == "__main__":
    main()
