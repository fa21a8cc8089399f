"""Compliance topology optimisation by the OC method on the GPU library.

No reference counterpart: the reference updates densities by a stress-ratio
heuristic (src/Optimization/TopOpt.jl:139-405).  This driver is the published
optimality-criteria loop (Bendsoe & Sigmund; the top88/top3d family) with the
Helmholtz PDE filter as density and sensitivity filter (the filter operator
F = (vol/64) S^T A^-1 S is symmetric, so F^T = F):

    rho = F(x)                       physical density
    factor = Emin + rho^p (E0-Emin)  SIMP modulus
    u: warm-started Jacobi-PCG solve of K(factor) u = f
    c = f.u;  dc = -p rho^(p-1) (E0-Emin) u_e^T Ke u_e
    dc_x = F(dc);  x <- OC(x, dc_x, dv=1, volfrac, move)

The bisection keeps sum(x_new) <= volfrac*nE on the design variables.

run_oc takes host arrays (each call copies through the C ABI); run_oc_device
keeps the whole iteration on the GPU (grid meshes) and can solve with the
mixed-precision and learned forms, fine-tuning the learned preconditioner
every few iterations on the current design.
"""
import time

import numpy as np

from ._lib import HX_OK, HX_NOT_CONVERGED, Context, default_opts


class OCResult:
    def __init__(self):
        self.compliance = []
        self.iterations = []
        self.change = []
        self.solve_ms = []
        self.x = None
        self.rho = None
        self.u = None


def run_oc(ctx: Context, bc_indicator, f, volfrac, radius, n_iter, p=3.0, e0=1.0, emin=1e-9,
           nu=0.3, move=0.2, tol=1e-6, ref_compat=0, filter_tol=1e-5, filter_max_iter=200,
           precision=0, max_iter=40000, callback=None):
    """Runs n_iter OC iterations on the mesh already set in ctx."""
    (nx, ny, nz), _ = ctx.grid()
    ne = nx * ny * nz
    ctx.set_material(1.0, nu)
    ctx.set_bc(bc_indicator)
    x = np.full(ne, float(volfrac))
    u = None
    res = OCResult()
    ones = np.ones(ne)
    for it in range(n_iter):
        rho, _ = ctx.filter(x, radius, ref_compat, filter_tol, filter_max_iter)
        fac = emin + np.power(np.clip(rho, 0.0, None), p) * (e0 - emin)
        opts = default_opts(tol=tol, max_iter=max_iter, precision=precision)
        t0 = time.perf_counter()
        u, rep = ctx.solve(f, fac, u0=u, opts=opts, ok=(HX_OK, HX_NOT_CONVERGED))
        res.solve_ms.append((time.perf_counter() - t0) * 1e3)
        c = ctx.compliance(f, u)
        ce = ctx.element_energy(u, ne)
        dc = -p * np.power(np.clip(rho, 0.0, None), p - 1) * (e0 - emin) * ce
        dcf, _ = ctx.filter(dc, radius, ref_compat, filter_tol, filter_max_iter)
        xn, lam, steps = ctx.oc_update(x, dcf, ones, volfrac, move)
        res.change.append(float(np.abs(xn - x).max()))
        res.compliance.append(c)
        res.iterations.append(rep.iterations)
        x = xn
        if callback:
            callback(it, c, rep)
    res.x, res.rho, res.u = x, rho, u
    return res


def run_oc_device(ctx: Context, bc_indicator, f, volfrac, radius, n_iter, p=3.0, e0=1.0,
                  emin=1e-9, nu=0.3, move=0.2, tol=1e-6, ref_compat=0, filter_tol=1e-5,
                  filter_max_iter=200, precision=0, preconditioner=0, max_iter=200000,
                  finetune_every=0, finetune_kw=None, adaptive=True, retry_every=20,
                  shift_factor=0.0, callback=None):
    """The OC loop of run_oc on device arrays (the mesh set by hx_set_grid):
    filter, SIMP, warm-started solve (precision / preconditioner as in
    hx_solve_opts), compliance, sensitivities, filtered sensitivities and the
    OC update all run on the GPU; only scalars come back.  With the learned
    preconditioner and finetune_every > 0 the networks are fine-tuned on the
    current design every finetune_every iterations (learned.finetune).

    adaptive (learned preconditioner only): the first solve uses Jacobi and
    its time and iteration count are kept; a learned solve may take at most
    that many iterations (a learned iteration costs more than a Jacobi one)
    and, if it has not converged by then, is finished by Jacobi-PCG from its
    iterate.  A learned solve slower than the latest Jacobi solve, or one
    that fell back or was finished by Jacobi, switches the following solves
    to Jacobi until the next fine-tuning or `retry_every` iterations later.
    On designs unlike its training data the networks can cost more than they
    save, and this keeps the loop near Jacobi's cost there.  res.pc_used
    records the choice per iteration.

    shift_factor: the regularisation shift of hx_solve_opts (the reference's
    solve_system_gpu default is 1e-6), needed when the supports leave a
    rigid mode free."""
    import importlib

    import torch
    (nx, ny, nz), _ = ctx.grid()
    ne = nx * ny * nz
    ctx.set_material(1.0, nu)
    ctx.set_bc(bc_indicator)
    dev = torch.device("cuda", torch.cuda.current_device())
    f_d = torch.from_numpy(np.ascontiguousarray(f, dtype=np.float64)).to(dev)
    x = torch.full((ne,), float(volfrac), dtype=torch.float64, device=dev)
    xn, rho, fac, dc, dcf = (torch.empty_like(x) for _ in range(5))
    u = torch.zeros_like(f_d)
    torch.cuda.current_stream().synchronize()
    learned = importlib.import_module(__package__ + ".learned") if finetune_every else None
    res = OCResult()
    res.finetune_ms = []
    res.pc_used = []
    res.fallback = []  # learned solves that fell back or were finished by Jacobi
    use_learned = preconditioner == 1 and not adaptive
    jac_ms = jac_its = None
    retry_at = 0
    for it in range(n_iter):
        if preconditioner == 1 and adaptive and not use_learned and jac_ms is not None \
                and it >= retry_at:
            use_learned = True
        pc = 1 if use_learned else (3 if preconditioner == 3 else 0)
        ctx.filter_device(x.data_ptr(), rho.data_ptr(), radius, ref_compat, filter_tol,
                          filter_max_iter)
        ctx.simp_device(rho.data_ptr(), fac.data_ptr(), p, e0, emin)
        cap = max_iter
        if pc == 1 and adaptive and jac_its is not None:
            cap = min(max_iter, max(jac_its, 50))
        opts = default_opts(tol=tol, max_iter=cap, precision=precision, preconditioner=pc,
                            warm_start=1 if it else 0, shift_factor=shift_factor)
        t0 = time.perf_counter()
        rep = ctx.solve_device(f_d.data_ptr(), fac.data_ptr(), u.data_ptr(), opts=opts,
                               ok=(HX_OK, HX_NOT_CONVERGED))
        finished_by_jacobi = False
        if pc == 1 and rep.status != HX_OK:
            opts = default_opts(tol=tol, max_iter=max_iter, precision=precision, preconditioner=0,
                                warm_start=1, shift_factor=shift_factor)
            rep2 = ctx.solve_device(f_d.data_ptr(), fac.data_ptr(), u.data_ptr(), opts=opts,
                                    ok=(HX_OK, HX_NOT_CONVERGED))
            rep2.iterations += rep.iterations
            rep, finished_by_jacobi = rep2, True
        ms = (time.perf_counter() - t0) * 1e3
        res.solve_ms.append(ms)
        res.pc_used.append(pc)
        res.fallback.append(int(pc == 1 and (bool(rep.fallback_used) or finished_by_jacobi)))
        if preconditioner == 1 and adaptive:
            if pc == 0:
                jac_ms, jac_its = ms, rep.iterations
            elif rep.fallback_used or finished_by_jacobi or (jac_ms is not None and ms > jac_ms):
                use_learned = False
                retry_at = it + retry_every
        c = ctx.compliance_device(f_d.data_ptr(), u.data_ptr())
        ctx.sensitivity_device(rho.data_ptr(), u.data_ptr(), dc.data_ptr(), p, e0, emin)
        ctx.filter_device(dc.data_ptr(), dcf.data_ptr(), radius, ref_compat, filter_tol,
                          filter_max_iter)
        ctx.oc_update_device(x.data_ptr(), dcf.data_ptr(), xn.data_ptr(), volfrac, move)
        res.change.append(float((xn - x).abs().max()))  # torch, then synchronised
        res.compliance.append(c)
        res.iterations.append(rep.iterations)
        x, xn = xn, x
        if callback:
            callback(it, c, rep)
        if learned and preconditioner == 1 and (it + 1) % finetune_every == 0 and it + 1 < n_iter:
            t1 = time.perf_counter()
            learned.finetune(ctx, f_d, fac, u, **(finetune_kw or {}))
            res.finetune_ms.append((time.perf_counter() - t1) * 1e3)
            retry_at = it + 1  # the fine-tuned networks get the next solve
    torch.cuda.current_stream().synchronize()
    res.x, res.rho, res.u = x.cpu().numpy(), rho.cpu().numpy(), u.cpu().numpy()
    return res
