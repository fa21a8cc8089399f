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
