"""Training and loading of the learned preconditioner.

The network and its training kernels live in the library (hx_net_*); this
module drives them.  It generates residual/error pairs from the library's
own Jacobi-PCG, on seeded problems built like the scale workload (i.i.d.
uniform element densities smoothed by the Helmholtz filter, mapped to
[1e-3, 1], SIMP p = 3) over a mixture of grid shapes, supports (cantilever,
MBB), filter radii and sharpened near-0/1 densities.  Per problem:
  1. solve to rtol 1e-11 for u*;
  2. record `snaps` Jacobi-PCG iterates x_k spread over a solve to rtol 1e-8;
  3. take `steps` Adam steps, each on the summed gradient of `batch` random
     pairs r = b - K x_k, e = u* - x_k (energy-norm loss).
The trained parameters are stored as a float32 .npy of HX_NET_PARAMS values.
"""
import os

import numpy as np

from . import workloads as W

WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "spd_cnn_mix.npy")


def problem(ctx, dims, seed, radius=3.0, support="cantilever", sharpen=0.0):
    """(f, fac) device tensors of one seeded problem; sets the grid and BCs.
    support: "cantilever" (clamped x = 0, line load) or "mbb" (half MBB beam).
    sharpen > 0 pushes the smoothed densities towards 0/1 like an optimised
    design: rho <- logistic(sharpen (rho - 0.5)) before the map to [1e-3, 1]."""
    import torch
    nx, ny, nz = dims
    if support == "mbb":
        _, _, bc, f = W.mbb_half_beam(nx, ny, nz, with_elements=False)
    else:
        _, _, bc, f = W.cantilever(nx, ny, nz, with_elements=False)
    ctx.set_grid(nx, ny, nz)
    ctx.set_material(1.0, 0.3)
    ctx.set_bc(bc)
    raw = W.raw_density(nx * ny * nz, seed)
    rho_f, _ = ctx.filter(raw, radius, 0, 1e-5, 200)
    if sharpen > 0:
        lo, hi = float(rho_f.min()), float(rho_f.max())
        t = (rho_f - lo) / max(hi - lo, 1e-30)
        rho_f = 1.0 / (1.0 + np.exp(-sharpen * (t - 0.5)))
    fac = W.simp(W.map_density(rho_f, 1e-3), 3.0, 1.0, 1e-9)
    dev = torch.device("cuda", torch.cuda.current_device())
    return torch.from_numpy(f).to(dev), torch.from_numpy(fac).to(dev)


# The training mixture: grid shapes from small slabs to the 128 x 64 x 64
# training grid (the networks act on coarse levels, whose meaning in
# physical scale depends on the grid), both supports, smooth and sharpened
# (near 0/1) densities, filter radii 1.5 - 4.
MIX_DIMS = [(128, 64, 64), (96, 48, 48), (64, 32, 32), (60, 20, 20), (96, 32, 32), (48, 24, 24),
            (80, 40, 20), (128, 48, 32)]


def mixture_case(k, rng):
    dims = MIX_DIMS[k % len(MIX_DIMS)]
    support = "mbb" if rng.random() < 0.4 else "cantilever"
    sharpen = float(rng.uniform(8.0, 30.0)) if rng.random() < 0.5 else 0.0
    radius = float(rng.uniform(1.5, 4.0))
    return dims, dict(radius=radius, support=support, sharpen=sharpen)


def _solve(ctx, hx, f, fac, **kw):
    import torch
    u = torch.zeros_like(f)
    rep = ctx.solve_device(f.data_ptr(), fac.data_ptr(), u.data_ptr(),
                           opts=hx.default_opts(**kw), ok=(0, 1, 3, 4, 9))
    return u, rep


def train(ctx, dims=None, problems=80, snaps=128, steps=150, batch=8, lr=(3e-4, 1e-4),
          seed0=1000, init_seed=5, log=None):
    """Train from a fresh initialisation; returns (params, losses).  dims:
    one grid for every problem, or None for the training mixture
    (mixture_case).  The learning rate steps from lr[0] to lr[1] halfway."""
    import importlib
    import torch
    hx = importlib.import_module(__package__)
    ctx.net_init(seed=init_seed)
    losses = []
    rng = np.random.default_rng(seed0)
    total = problems * steps
    for p in range(problems):
        if dims is None:
            d, kw = mixture_case(p, rng)
        else:
            d, kw = dims, {}
        f, fac = problem(ctx, d, seed0 + p, **kw)
        n = f.numel()
        u_star, _ = _solve(ctx, hx, f, fac, tol=1e-11, max_iter=1000000)
        _, rj = _solve(ctx, hx, f, fac, tol=1e-8, max_iter=1000000)
        every = max(2, 2 * int(np.ceil(rj.iterations / (2.0 * snaps))))
        X = torch.zeros((snaps, n), dtype=torch.float64, device=f.device)
        taken = ctx.pcg_snapshots(f.data_ptr(), fac.data_ptr(), every, snaps, 1e-8, X.data_ptr())
        ctx.net_prepare(fac.data_ptr())
        R = torch.empty((batch, n), dtype=torch.float64, device=f.device)
        E = torch.empty_like(R)
        for s in range(steps):
            ks = rng.integers(taken, size=batch)
            for b, k in enumerate(ks):
                ctx.residual_device(f.data_ptr(), fac.data_ptr(), X[k].data_ptr(), R[b].data_ptr())
                torch.sub(u_star, X[k], out=E[b])
            torch.cuda.current_stream().synchronize()
            rate = lr[0] if len(losses) < total // 2 else lr[1]
            losses.append(ctx.net_train_batch([R[b].data_ptr() for b in range(batch)],
                                              [E[b].data_ptr() for b in range(batch)], rate, 0))
        if log:
            log(f"problem {p} {d} {kw}: jacobi {rj.iterations} its to 1e-8, {taken} snapshots, "
                f"loss {np.mean(losses[-steps:]):.4f}")
        del X, R, E
    return ctx.net_get_params(), np.array(losses)


def finetune(ctx, f_d, fac_d, u_star, steps=40, batch=4, lr=1e-4, snaps=16, every=64,
             snap_tol=1e-3, seed=0):
    """Fine-tunes the loaded networks on the current system (device f, factors,
    and its solution u_star, e.g. the last solve to rtol 1e-6): `snaps`
    Jacobi-PCG iterates every `every` iterations up to rtol snap_tol, then
    `steps` Adam steps on batches of (r, e = u_star - x_k) pairs.  The Adam
    moments restart (hx_net_set_params)."""
    import torch
    n = f_d.numel()
    ctx.net_set_params(ctx.net_get_params())
    X = torch.zeros((snaps, n), dtype=torch.float64, device=f_d.device)
    torch.cuda.current_stream().synchronize()
    taken = ctx.pcg_snapshots(f_d.data_ptr(), fac_d.data_ptr(), every, snaps, snap_tol,
                              X.data_ptr())
    ctx.net_prepare(fac_d.data_ptr())
    rng = np.random.default_rng(seed)
    R = torch.empty((batch, n), dtype=torch.float64, device=f_d.device)
    E = torch.empty_like(R)
    losses = []
    for _ in range(steps):
        ks = rng.integers(taken, size=batch)
        for b, k in enumerate(ks):
            ctx.residual_device(f_d.data_ptr(), fac_d.data_ptr(), X[k].data_ptr(), R[b].data_ptr())
            torch.sub(u_star, X[k], out=E[b])
        torch.cuda.current_stream().synchronize()
        losses.append(ctx.net_train_batch([R[b].data_ptr() for b in range(batch)],
                                          [E[b].data_ptr() for b in range(batch)], lr, 0))
    del X, R, E
    return np.array(losses)


def save_params(path, params):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.save(path, np.asarray(params, np.float32))


def load_params(path=DEFAULT_WEIGHTS):
    p = np.load(path)
    if p.dtype != np.float32 or p.ndim != 1:
        raise ValueError(f"{path}: expected a flat float32 array")
    return p


def load_into(ctx, path=DEFAULT_WEIGHTS):
    """Load trained parameters into the context's network."""
    ctx.net_set_params(load_params(path))


def main(argv=None):
    """Regenerate the default weights: python -m <package>.learned [--out PATH]."""
    import argparse
    import importlib
    import time
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--problems", type=int, default=80)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=3e-4)
    a = ap.parse_args(argv)
    hx = importlib.import_module(__package__)
    t0 = time.time()
    with hx.Context(0) as ctx:
        params, losses = train(ctx, problems=a.problems, steps=a.steps, batch=a.batch,
                               lr=(a.lr, a.lr / 3),
                               log=lambda m: print(f"[{time.time() - t0:.0f}s] {m}", flush=True))
    save_params(a.out, params)
    print(f"{len(losses)} Adam steps, loss {losses[:50].mean():.4f} -> {losses[-50:].mean():.4f}; "
          f"saved {a.out}")


if __name__ == "__main__":
    main()
