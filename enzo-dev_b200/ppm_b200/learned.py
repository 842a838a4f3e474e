"""Training of the learned Newton start (the 6 -> 64 -> 64 -> 1 MLP of ppm_guess.cuh).

Pipeline, every numeric step in the library's own CUDA kernels:
  1. run the plain solver with Riemann logging on (ppm_b200_riemann_log): the Sod tube
     (64^3, gamma 1.4, 100 steps) and the decaying Mach-3 turbulence (256^3, gamma 5/3,
     50 steps); each log record holds a face's states and its converged p*;
  2. turn records into samples (ppm_b200_guess_features): the 6 normalised inputs and
     the target r = ln(p* / p_acoustic) / |x|^2;
  3. minibatch Adam (ppm_b200_guess_grad forward + backward, ppm_b200_guess_adam).
torch only holds the device buffers and draws the minibatch permutations; the context
should run on torch's current stream (Context(0, stream=...)), and the functions below
also synchronise wherever torch prepares data that the library reads.

    python -m ppm_b200.learned --out enzo-dev_b200/ppm_b200/guess_weights.npy
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

from . import capi
from . import harness as H

NWEIGHTS = capi.GUESS_WEIGHTS
WEIGHTS_FILE = Path(__file__).resolve().parent / "guess_weights.npy"


def init_weights(seed=0):
    """He-style initial weights: W1[6][64] b1 W2[64][64] b2 w3 b3."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NWEIGHTS, dtype=np.float32)
    w[0:384] = rng.standard_normal(384) * np.sqrt(2.0 / 6)
    w[448:4544] = rng.standard_normal(4096) * np.sqrt(2.0 / 64)
    w[4608:4672] = rng.standard_normal(64) * np.sqrt(1.0 / 64)
    return w


def default_weights():
    """The committed weights trained by this module's CLI."""
    return np.load(WEIGHTS_FILE).astype(np.float32)


def _sod(hp, n):
    g = H.Grid.uniform((n, n, n))
    f = H.shock_tube(g, hp, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    H.fill_ghosts(g, f, "outflow")
    return g, f, ("outflow",) * 3


def _turbulence(hp, n, mach, seed):
    g = H.Grid.uniform((n, n, n))
    return g, H.turbulence(g, hp, mach=mach, seed=seed), ("periodic",) * 3


def run_steps(ctx, g, fields_host, hp, steps, bc, learned=False, torch=None):
    """Advance a grid on the device (time step, SolvePPM_DE, ghost fill); returns the
    device fields and the summed stats."""
    dev = torch.device("cuda", torch.cuda.current_device())
    f = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in fields_host.items()}
    dtd = torch.zeros(1, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    tot = None
    for cyc in range(steps):
        ctx.compute_timestep(g, hp, f, memory=capi.MEM_DEVICE, dt_device=dtd, want_host=False)
        rc, st = ctx.solve_ppm_de(g, hp, 0.0, cyc, f, memory=capi.MEM_DEVICE, want_stats=True,
                                  dt_device=dtd, learned_guess=learned)
        tot = st if tot is None else {k: (tot[k] + st[k] if not isinstance(st[k], list) else
                                          [a + b for a, b in zip(tot[k], st[k])]) for k in st}
        ctx.set_boundary(g, f, hp.dual, bc)
    return f, tot


def collect(ctx, torch, stride_sod=64, stride_turb=256, capacity=12_000_000, sod_n=64,
            turb_n=256, sod_steps=100, turb_steps=50, log=print):
    """Log Riemann problems of the plain solver on the two training workloads; returns
    device samples (n, 8) with only usable rows."""
    out = []
    for name, make, hp, steps, stride in (
        ("sod", lambda hp: _sod(hp, sod_n), H.HydroParams(gamma=1.4, cfl=0.4, dual=True),
         sod_steps, stride_sod),
        ("turbulence", lambda hp: _turbulence(hp, turb_n, 3.0, 1234),
         H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True), turb_steps, stride_turb),
    ):
        g, f, bc = make(hp)
        rec = torch.zeros((capacity, 8), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        ctx.riemann_log(rec, stride)
        run_steps(ctx, g, f, hp, steps, bc, torch=torch)
        n = ctx.riemann_log_count()
        ctx.riemann_log(None, 0)
        s = torch.zeros((max(n, 1), 8), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.guess_features(rec, n, hp.gamma, hp.tiny_number, s)
        torch.cuda.synchronize()
        s = s[:n]
        s = s[s[:, 7] > 0]
        log(f"[collect] {name}: {n} records, {s.shape[0]} usable samples")
        out.append(s)
        del rec
    return torch.cat(out, 0)


def train(ctx, torch, samples, epochs=12, batch=65536, lr=2e-3, seed=0, log=print):
    """Minibatch Adam on device samples; returns (weights, per-epoch mean losses)."""
    dev = samples.device
    w = torch.from_numpy(init_weights(seed)).to(dev)
    grad = torch.zeros(NWEIGHTS, dtype=torch.float32, device=dev)
    m = torch.zeros_like(grad)
    v = torch.zeros_like(grad)
    loss = torch.zeros(1, dtype=torch.float64, device=dev)
    n = samples.shape[0]
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    step = 0
    history = []
    for ep in range(epochs):
        perm = torch.randperm(n, device=dev, generator=gen)
        loss.zero_()
        torch.cuda.synchronize()
        lr_ep = lr * (0.5 * (1.0 + np.cos(np.pi * ep / epochs)))  # cosine decay
        for s0 in range(0, n, batch):
            idx = perm[s0:s0 + batch]
            nb = idx.shape[0]
            ctx.guess_grad(w, samples, idx, nb, grad, loss)
            step += 1
            ctx.guess_adam(w, grad, m, v, step, lr_ep)
        torch.cuda.synchronize()
        history.append(float(loss.item()) / n)
        log(f"[train] epoch {ep}: mse {history[-1]:.4e}")
    return w.cpu().numpy(), history


def evaluate(ctx, torch, weights, n=128, mach=10.0, steps=3, seed=77, log=print):
    """Newton iterations per interface and time per step, plain vs learned start, on
    periodic turbulence (the generator of the training data, rms Mach `mach`)."""
    hp = H.HydroParams(gamma=5.0 / 3.0, cfl=0.4, dual=True)
    g, f, bc = _turbulence(hp, n, mach, seed)
    ctx.set_guess(weights)
    res = {}
    for learned in (False, True):
        run_steps(ctx, g, f, hp, 1, bc, learned=learned, torch=torch)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, st = run_steps(ctx, g, f, hp, steps, bc, learned=learned, torch=torch)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        key = "learned" if learned else "plain"
        res[key] = {"newton_per_interface": st["newton_iters"] / st["interfaces"],
                    "rejected": st["guess_rejected"], "s_per_step": el / steps}
        log(f"[eval] {key}: {res[key]}")
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(WEIGHTS_FILE))
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--stride-turb", type=int, default=256)
    ap.add_argument("--stride-sod", type=int, default=64)
    ap.add_argument("--turb-n", type=int, default=256)
    ap.add_argument("--report", default=None, help="write a JSON summary here")
    args = ap.parse_args(argv)
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = capi.Context(0, stream=stream.cuda_stream)
    t0 = time.perf_counter()
    samples = collect(ctx, torch, stride_sod=args.stride_sod, stride_turb=args.stride_turb,
                      turb_n=args.turb_n)
    t1 = time.perf_counter()
    w, hist = train(ctx, torch, samples, epochs=args.epochs, batch=args.batch, lr=args.lr)
    t2 = time.perf_counter()
    np.save(args.out, w)
    ev = evaluate(ctx, torch, w)
    rep = {"samples": int(samples.shape[0]), "collect_s": t1 - t0, "train_s": t2 - t1,
           "epochs": args.epochs, "batch": args.batch, "lr": args.lr, "mse": hist, "eval": ev}
    print(json.dumps(rep))
    if args.report:
        Path(args.report).write_text(json.dumps(rep, indent=1))
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
