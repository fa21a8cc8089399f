"""The geometric multigrid preconditioner (hx_gmg.cu, HX_PC_MULTIGRID): the
GPU replacement of the reference's CPU AMG (src/Solvers/GPUSolver.jl:
168-268, 513-516).  Its flexible-CG solve must reach the oracle's solution
and take far fewer iterations than Jacobi-PCG; with the reference's failure
handling ("jacobi_amg", GPUSolver.jl:540-579) a stagnated Jacobi attempt
hands over to it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(ctx, hx, dims, seed=7, lo=1e-3):
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    ctx.set_grid(*dims)
    ctx.set_material(1.0, 0.3)
    ctx.set_bc(bc)
    rho_raw = hx.workloads.splitmix64_uniform(seed, el.shape[0])
    rho_f, _ = ctx.filter(rho_raw, 2.0, 0)
    rho = hx.workloads.map_density(rho_f, lo)
    return nodes, el, bc, f, hx.workloads.simp(rho)


@pytest.mark.parametrize("dims", [(64, 16, 16), (96, 32, 32)])
def test_multigrid_fcg_matches_oracle(ctx, hx, orc, dims):
    nodes, el, bc, f, fac = _problem(ctx, hx, dims)
    uj, rj = ctx.solve(f, fac, tol=1e-8, max_iter=100000)
    um, rm = ctx.solve(f, fac, tol=1e-8, max_iter=100000, preconditioner=3)
    assert rm.status == 0 and rm.true_rel_res < 1e-8, rm.as_dict()
    # fewer iterations than Jacobi-PCG by a wide margin
    assert rm.iterations * 3 < rj.iterations, (rm.iterations, rj.iterations)
    c0 = hx.mesh.connectivity0(el)
    ke = orc.canonical_ke()
    free = orc.free_mask_from(bc, orc.diagonal(c0, nodes.shape[0], ke, fac))
    ku = orc.apply_stiffness(c0, nodes.shape[0], ke, fac, um)
    b = f * free
    assert np.linalg.norm((b - ku) * free) / np.linalg.norm(b) < 1e-8
    assert np.abs(um - uj).max() <= 1e-5 * np.abs(uj).max()
    c_m, c_j = float(f @ um), float(f @ uj)
    assert abs(c_m - c_j) <= 1e-8 * abs(c_j)


def test_multigrid_takes_over_from_stagnated_jacobi(ctx, hx):
    """ref_retry with multigrid_fallback: Jacobi-PCG stopped by max_iter in
    the (5e-2, 0.1] band is not accepted as stagnation when a stronger
    preconditioner is available; attempt 2 runs multigrid with the shift
    escalated x10, as the reference's jacobi_amg switches to AMG."""
    dims = (10, 4, 4)
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    rng = np.random.default_rng(3)
    fac = hx.workloads.simp(rng.uniform(0.2, 1.0, el.shape[0]))
    ctx.set_grid(*dims)
    ctx.set_material(1.0, 0.3)
    ctx.set_bc(bc)
    u, rep = ctx.solve(f, fac, tol=1e-8, max_iter=110, shift_factor=1e-9, ref_retry=1,
                       keep_best=1, multigrid_fallback=1, ok=(0, 1, 2))
    assert rep.status == 0 and rep.attempts == 2 and rep.fallback_used == 1, rep.as_dict()
    # attempt 2 solved the system with the shift escalated x10 (1e-8 x max diag)
    uj, rj = ctx.solve(f, fac, tol=1e-11, shift_factor=1e-8)
    assert np.abs(u - uj).max() <= 1e-5 * np.abs(uj).max()
    # without the fallback a stagnation below 5e-2 is accepted on attempt 1
    _, r2 = ctx.solve(f, fac, tol=1e-8, max_iter=127, shift_factor=1e-9, ref_retry=1,
                      keep_best=1, ok=(0, 1, 2))
    assert r2.status == 2 and r2.attempts == 1


def test_reference_shaped_solve_reports_gmg(ctx, hx):
    from importlib import import_module
    api = import_module("2025_12_09_hexat_v069_b200.api")
    dims = (10, 4, 4)
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    dens = np.random.default_rng(3).uniform(0.2, 1.0, el.shape[0]).astype(np.float32)
    x, rel, name = api.solve_system_gpu(nodes, el, 1.0, 0.3, bc, f.astype(np.float32), dens,
                                        max_iter=60, tol=1e-7, shift_factor=1e-9, ctx=ctx)
    assert name == "GMG" and rel < 1e-7


def test_vcycle_is_a_symmetric_linear_operator(ctx, hx):
    """hx_gmg_apply after a multigrid solve: the V-cycle (Chebyshev smoothing
    on a Lanczos lambda_max, direct coarsest solve) is linear and symmetric
    up to FP32 rounding, positive on the free DOFs, and zero on the fixed
    ones -- what flexible CG needs from a preconditioner."""
    import torch
    dims = (64, 16, 16)
    nodes, el, bc, f, fac = _problem(ctx, hx, dims)
    dev = torch.device("cuda", 0)
    f_d = torch.from_numpy(f).to(dev)
    fac_d = torch.from_numpy(fac).to(dev)
    u = torch.zeros_like(f_d)
    rep = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u.data_ptr(),
                           opts=hx.default_opts(tol=1e-8, preconditioner=3))
    assert rep.status == 0 and rep.iterations < 40, rep.as_dict()
    free = torch.from_numpy(bc.reshape(-1) == 0).to(dev)
    g = torch.Generator(device="cpu").manual_seed(0)
    r = [torch.randn(f_d.numel(), generator=g, dtype=torch.float64).to(dev) * free
         for _ in range(2)]
    z = []
    for v in r:
        out = torch.empty_like(v)
        ctx.gmg_apply(v.data_ptr(), out.data_ptr())
        z.append(out)
    # (each call waits for the default stream, where torch wrote r)
    a, b = float(r[0] @ z[1]), float(r[1] @ z[0])
    scale = np.sqrt(float(r[0] @ z[0]) * float(r[1] @ z[1]))
    assert float(r[0] @ z[0]) > 0 and float(r[1] @ z[1]) > 0
    assert abs(a - b) <= 1e-5 * scale, (a, b)
    out = torch.empty_like(r[0])
    ctx.gmg_apply((2 * r[0] + r[1]).data_ptr(), out.data_ptr())
    ref = 2 * z[0] + z[1]
    assert float(torch.linalg.norm(out - ref) / torch.linalg.norm(ref)) < 1e-5
    assert not torch.any(z[0][~free])


def test_mixed_precision_multigrid_fcg(ctx, hx, orc):
    """FP32 flexible CG with FP64 reliable updates around the V-cycle reaches
    the FP64 true residual and the oracle's solution."""
    dims = (64, 16, 16)
    nodes, el, bc, f, fac = _problem(ctx, hx, dims)
    uj, rj = ctx.solve(f, fac, tol=1e-10, max_iter=100000)
    um, rm = ctx.solve(f, fac, tol=1e-8, max_iter=100000, precision=1, preconditioner=3)
    assert rm.status == 0 and rm.true_rel_res < 1e-8 and rm.fallback_used == 0, rm.as_dict()
    assert rm.iterations < 60, rm.as_dict()
    c0 = hx.mesh.connectivity0(el)
    ke = orc.canonical_ke()
    free = orc.free_mask_from(bc, orc.diagonal(c0, nodes.shape[0], ke, fac))
    ku = orc.apply_stiffness(c0, nodes.shape[0], ke, fac, um)
    b = f * free
    assert np.linalg.norm((b - ku) * free) / np.linalg.norm(b) < 1e-8
    assert np.abs(um - uj).max() <= 1e-5 * np.abs(uj).max()


@pytest.mark.parametrize("precision", [0, 1])
def test_multigrid_on_a_shifted_singular_system(ctx, hx, precision):
    """The MBB half-beam's supports leave the rigid z-translation free, so K
    is singular and the solve needs the shift (1e-6 x max diag, the
    reference's default).  The coarse levels carry the shift seen through
    the transfers (8x per level), so they and the dense coarsest inverse stay
    nonsingular: the multigrid solve converges in few iterations to the
    Jacobi-PCG solution of the same shifted system."""
    dims = (32, 16, 16)
    nodes, el, bc, f = hx.workloads.mbb_half_beam(*dims)
    rng = np.random.default_rng(11)
    fac = hx.workloads.simp(rng.uniform(0.1, 1.0, el.shape[0]))
    ctx.set_grid(*dims)
    ctx.set_material(1.0, 0.3)
    ctx.set_bc(bc)
    uj, rj = ctx.solve(f, fac, tol=1e-10, max_iter=200000, shift_factor=1e-6)
    um, rm = ctx.solve(f, fac, tol=1e-8, max_iter=2000, shift_factor=1e-6, precision=precision,
                       preconditioner=3)
    assert rm.status == 0 and rm.true_rel_res < 1e-8 and rm.fallback_used == 0, rm.as_dict()
    assert rm.iterations < 60, rm.as_dict()
    assert np.abs(um - uj).max() <= 1e-5 * np.abs(uj).max()


def test_smoothing_degree_option(ctx, hx):
    """mg_smooth_degree selects the Chebyshev degree (odd degrees end the
    buffer alternation on the other buffer, which the smoother corrects):
    every degree 1..4 converges to the same solution; out-of-range values are
    rejected before any work."""
    dims = (48, 16, 16)
    nodes, el, bc, f, fac = _problem(ctx, hx, dims)
    us = []
    for deg in (1, 2, 3, 4):
        u, rep = ctx.solve(f, fac, tol=1e-9, max_iter=500, preconditioner=3,
                           mg_smooth_degree=deg)
        assert rep.status == 0 and rep.true_rel_res < 1e-9, (deg, rep.as_dict())
        us.append(u)
    for u in us[1:]:
        assert np.abs(u - us[0]).max() <= 1e-6 * np.abs(us[0]).max()
    with pytest.raises(hx.HexatError) as err:
        ctx.solve(f, fac, tol=1e-9, preconditioner=3, mg_smooth_degree=9)
    assert err.value.status == 6  # HX_BAD_ARG


def test_dropin_solve_with_multigrid_selected(ctx, hx):
    """hx_set_dropin_solver, and the reference's config key that selects it
    (solver_parameters.preconditioner = "amg"): the reference-shaped
    solve_system_gpu runs the multigrid-preconditioned solve from its first
    attempt (prec_name "GMG") and returns the Jacobi drop-in's solution
    within the tolerances of both solves; "jacobi_amg" brings back the
    default."""
    from importlib import import_module
    api = import_module("2025_12_09_hexat_v069_b200.api")
    dims = (40, 12, 12)
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    dens = np.random.default_rng(5).uniform(0.2, 1.0, el.shape[0]).astype(np.float32)
    args = (nodes, el, 1.0, 0.3, bc, f.astype(np.float32), dens)
    amg = {"solver_parameters": {"preconditioner": "amg"}}
    default = {"solver_parameters": {"preconditioner": "jacobi_amg"}}
    try:
        xj, rj, nj = api.solve_system_gpu(*args, tol=1e-7, ctx=ctx)
        xm, rm, nm = api.solve_system_gpu(*args, tol=1e-7, config=amg, ctx=ctx)
        ctx.set_dropin_solver(3, 1, 0)  # mixed precision multigrid
        xq, rq, nq = api.solve_system_gpu(*args, tol=1e-7, ctx=ctx)
    finally:
        ctx.set_dropin_solver(0, 0, 1)
    assert nj == "Jacobi" and nm == "GMG" and nq == "GMG"
    assert rj < 1e-7 and rm < 1e-7 and rq < 1e-7
    scale = np.abs(xj).max()
    assert np.abs(xm - xj).max() <= 1e-4 * scale and np.abs(xq - xj).max() <= 1e-4 * scale
    _, _, n0 = api.solve_system_gpu(*args, tol=1e-7, config=default, ctx=ctx)
    assert n0 == "Jacobi"
    with pytest.raises(hx.HexatError):
        ctx.set_dropin_solver(2, 0, 0)  # HX_PC_NONE is not a drop-in choice
