"""Parity of the CUDA library (through the C ABI) with the CPU FP64 oracle.

Tolerances: the library and the oracle run the same FP64 algorithms with
different summation orders, so operator results agree to 1e-12 relative,
converged solves to a few times the requested tolerance, and the filter (same
Jacobi-CG, residual tested every 10 iterations) to 1e-9.  FP32 caller arrays
are compared at FP32 resolution (1e-5 relative).
"""
import numpy as np
import pytest

from tests.helpers import prune_system, reconstruct_full_solution

pytestmark = pytest.mark.gpu

GRIDS = [(1, 1, 1), (13, 7, 5), (40, 9, 17), (33, 2, 3), (64, 15, 8)]


def _setup(ctx, hx, dims, nu=0.3):
    nodes, el, _ = hx.mesh.generate_mesh(*dims)
    ctx.set_grid(*dims)
    ctx.set_material(1.0, nu)
    return nodes, el, hx.mesh.connectivity0(el)


@pytest.mark.parametrize("dims", GRIDS)
def test_apply_stiffness(ctx, hx, orc, dims):
    nodes, el, c0 = _setup(ctx, hx, dims)
    rng = np.random.default_rng(sum(dims))
    fac = rng.uniform(0.0, 1.0, c0.shape[0])
    fac[rng.uniform(size=fac.shape) < 0.2] = 0.0
    x = rng.standard_normal(3 * nodes.shape[0])
    y = ctx.apply_stiffness(x, fac)
    yo = orc.apply_stiffness(c0, nodes.shape[0], orc.canonical_ke(), fac, x)
    assert np.abs(y - yo).max() <= 1e-12 * max(1.0, np.abs(yo).max())


def test_apply_stiffness_box_elements(ctx, hx, orc):
    dims = (9, 6, 5)
    nodes, el, c0 = _setup(ctx, hx, dims, nu=0.27)
    ctx.set_grid(*dims, 1.3, 0.7, 2.1)
    ctx.set_material(1.0, 0.27)
    rng = np.random.default_rng(5)
    fac = rng.uniform(0.0, 1.0, c0.shape[0])
    x = rng.standard_normal(3 * nodes.shape[0])
    ke = orc.canonical_ke(1.3, 0.7, 2.1, 0.27)
    yo = orc.apply_stiffness(c0, nodes.shape[0], ke, fac, x)
    y = ctx.apply_stiffness(x, fac)
    assert np.abs(y - yo).max() <= 1e-12 * np.abs(yo).max()


def test_apply_stiffness_fp32_io(ctx, hx, orc):
    nodes, el, c0 = _setup(ctx, hx, (17, 5, 6))
    rng = np.random.default_rng(6)
    fac = rng.uniform(0.0, 1.0, c0.shape[0]).astype(np.float32)
    x = rng.standard_normal(3 * nodes.shape[0]).astype(np.float32)
    y = ctx.apply_stiffness(x, fac)
    assert y.dtype == np.float32
    yo = orc.apply_stiffness(c0, nodes.shape[0], orc.canonical_ke(), fac, x)
    assert np.abs(y - yo).max() <= 1e-5 * np.abs(yo).max()


def test_diagonal(ctx, hx, orc):
    nodes, el, c0 = _setup(ctx, hx, (11, 6, 4))
    fac = np.random.default_rng(7).uniform(0, 1, c0.shape[0])
    d = ctx.diagonal(fac, 3 * nodes.shape[0])
    do = orc.diagonal(c0, nodes.shape[0], orc.canonical_ke(), fac)
    assert np.abs(d - do).max() <= 1e-13 * do.max()


def test_operator_properties_full_size(ctx, hx):
    """At the 320x160x160 (8.2M element) size: linearity, symmetry and the
    rigid-body null space, checked through size-independent identities."""
    dims = (320, 160, 160)
    ctx.set_grid(*dims)
    ctx.set_material(1.0, 0.3)
    nn = 321 * 161 * 161
    rng = np.random.default_rng(8)
    fac = rng.uniform(1e-3, 1.0, 320 * 160 * 160)
    x1 = rng.standard_normal(3 * nn)
    x2 = rng.standard_normal(3 * nn)
    y1 = ctx.apply_stiffness(x1, fac)
    y2 = ctx.apply_stiffness(x2, fac)
    y12 = ctx.apply_stiffness(2.0 * x1 - 3.0 * x2, fac)
    assert np.abs(y12 - (2.0 * y1 - 3.0 * y2)).max() <= 1e-12 * np.abs(y12).max()
    a, b = np.dot(x2, y1), np.dot(x1, y2)
    assert abs(a - b) <= 1e-11 * abs(a)
    t = np.tile([0.3, -1.0, 2.0], nn)
    assert np.abs(ctx.apply_stiffness(t, fac)).max() <= 1e-12 * np.abs(y1).max()


def _cantilever(ctx, hx, dims, seed=11, contrast=True):
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    ctx.set_grid(*dims)
    ctx.set_material(1.0, 0.3)
    ctx.set_bc(bc)
    rho = np.random.default_rng(seed).uniform(0.05 if contrast else 0.5, 1.0, el.shape[0])
    fac = hx.workloads.simp(rho)
    return nodes, el, bc, f, fac


def test_solve_matches_oracle(ctx, hx, orc):
    dims = (16, 6, 6)
    nodes, el, bc, f, fac = _cantilever(ctx, hx, dims)
    c0 = hx.mesh.connectivity0(el)
    ke = orc.canonical_ke()
    nN = nodes.shape[0]
    free = orc.free_mask_from(bc, orc.diagonal(c0, nN, ke, fac))
    uo, ito, relo, _ = orc.cg_solve(c0, nN, ke, fac, free, f * free, tol=1e-10)
    u, rep = ctx.solve(f, fac, tol=1e-10)
    assert rep.status == 0 and rep.rel_res < 1e-10 and rep.true_rel_res < 5e-10
    assert abs(rep.iterations - ito) <= 3
    assert np.abs(u - uo).max() <= 1e-8 * np.abs(uo).max()
    assert np.all(u[free == 0] == 0)


def test_solve_shift_matches_oracle(ctx, hx, orc):
    dims = (12, 4, 5)
    nodes, el, bc, f, fac = _cantilever(ctx, hx, dims)
    c0 = hx.mesh.connectivity0(el)
    ke = orc.canonical_ke()
    nN = nodes.shape[0]
    free = orc.free_mask_from(bc, orc.diagonal(c0, nN, ke, fac))
    uo, ito, relo, sho = orc.cg_solve(c0, nN, ke, fac, free, f * free, tol=1e-9,
                                      shift_factor=1e-4, precond_add=True)
    u, rep = ctx.solve(f, fac, tol=1e-9, shift_factor=1e-4)
    assert rep.shift == pytest.approx(sho, rel=1e-12)
    assert abs(rep.iterations - ito) <= 2
    assert np.abs(u - uo).max() <= 1e-7 * np.abs(uo).max()


def test_solve_edge_cases(ctx, hx):
    dims = (10, 4, 4)
    nodes, el, bc, f, fac = _cantilever(ctx, hx, dims, contrast=False)
    u, rep = ctx.solve(f, fac, tol=1e-8)
    # warm start from the solution: converges at once
    u2, rep2 = ctx.solve(f, fac, u0=u, tol=1e-6)
    assert rep2.iterations <= 2 and np.abs(u2 - u).max() <= 1e-6 * np.abs(u).max()
    # zero right-hand side: zeros, "None" preconditioner semantics
    z, rz = ctx.solve(np.zeros_like(f), fac)
    assert rz.zero_rhs == 1 and np.all(z == 0)
    # iteration limit
    _, r3 = ctx.solve(f, fac, max_iter=3, ok=(1,))
    assert r3.status == 1 and r3.iterations == 3
    # NaN in the load: reported, not hung
    fn = f.copy()
    fn[5] = np.nan
    _, r4 = ctx.solve(fn, fac, ok=(4,))
    assert r4.status == 4
    # precision codes other than FP64 (0) and FP32-in-FP64 (1) are refused
    _, r5 = ctx.solve(f, fac, precision=2, ok=(6,))
    # a grid whose z-plane holds 3 x nodes >= 2^31 DOFs is refused by the
    # host check (32-bit in-plane offsets), before anything is allocated
    assert ctx.lib.hx_set_grid(ctx.h, 30000, 30000, 1, 1.0, 1.0, 1.0) == 6


def test_solve_deterministic(ctx, hx):
    dims = (20, 7, 9)
    nodes, el, bc, f, fac = _cantilever(ctx, hx, dims)
    u1, r1 = ctx.solve(f, fac, tol=1e-7)
    u2, r2 = ctx.solve(f, fac, tol=1e-7)
    assert r1.iterations == r2.iterations
    assert np.array_equal(u1, u2)


def test_mixed_precision(ctx, hx):
    dims = (24, 8, 8)
    nodes, el, bc, f, fac = _cantilever(ctx, hx, dims)
    u64, r64 = ctx.solve(f, fac, tol=1e-10)
    u, rep = ctx.solve(f, fac, tol=1e-6, precision=1)
    assert rep.status == 0 and rep.true_rel_res < 1e-6 and rep.refinements >= 1
    assert np.abs(u - u64).max() <= 1e-4 * np.abs(u64).max()
    c64, c = np.dot(f, u64), np.dot(f, u)
    assert abs(c - c64) <= 1e-5 * abs(c64)


@pytest.mark.parametrize("ref_compat", [0, 1])
@pytest.mark.parametrize("radius", [1.5, 3.0])
def test_filter_matches_oracle(ctx, hx, orc, ref_compat, radius):
    dims = (23, 11, 9)
    nodes, el, c0 = _setup(ctx, hx, dims)
    rho = hx.workloads.splitmix64_uniform(99, c0.shape[0])
    got, rep = ctx.filter(rho, radius, ref_compat, tol=1e-5)
    want, it, rel = orc.helmholtz_filter(c0, nodes.shape[0], rho, 1, 1, 1, radius, ref_compat,
                                         tol=1e-5)
    assert rep.iterations == it and rep.iterations % 10 == 0
    assert rep.rel_res == pytest.approx(rel, rel=1e-6)
    assert np.abs(got - want).max() <= 1e-10


def test_apply_gpu_filter_reference_shaped(ctx, hx, orc):
    from importlib import import_module
    api = import_module("2025_12_09_hexat_v069_b200.api")
    dims = (15, 6, 7)
    nodes, el, _ = hx.mesh.generate_mesh(*dims)
    c0 = hx.mesh.connectivity0(el)
    rho = hx.workloads.splitmix64_uniform(5, c0.shape[0]).astype(np.float32)
    out, t, it, res = api.apply_gpu_filter(rho, *dims, 1.0, 1.0, 1.0, 1.2, el, 1e-5, ctx=ctx)
    want, ito, _ = orc.helmholtz_filter(c0, nodes.shape[0], rho, 1, 1, 1, 1.2, 1, tol=1e-5)
    assert out.dtype == np.float32 and it == ito
    assert np.abs(out - want).max() <= 1e-6
    # a constant field comes back scaled by 1/1.5 (the reference element quirk)
    c, _, _, _ = api.apply_gpu_filter(np.full(c0.shape[0], 0.6, np.float32), *dims, 1.0, 1.0,
                                      1.0, 1.2, el, 1e-7, ctx=ctx)
    assert np.abs(c - 0.4).max() < 1e-5


def test_stress_matches_oracle(ctx, hx, orc):
    dims = (9, 7, 4)
    nodes, el, c0 = _setup(ctx, hx, dims)
    rng = np.random.default_rng(12)
    u = rng.standard_normal(3 * nodes.shape[0]) * 1e-2
    dens = rng.uniform(0, 1, c0.shape[0])
    dens[::7] = 1e-7
    got = ctx.stress(u, dens, 2.0, 0.3)
    want = orc.stress(c0, nodes, u, 2.0, 0.3, dens)
    for g, w in zip(got[:4], want[:4]):
        assert np.abs(g - w).max() <= 1e-12 * max(1e-30, np.abs(w).max())
    pr = want[0]
    gap = np.minimum(pr[:, 0] - pr[:, 1], 1e300)
    ok = gap > 1e-6 * np.abs(pr).max(1)
    assert np.abs(got[4][ok] - want[4][ok]).max() <= 1e-8
    assert np.all(got[0][::7] == 0)


def test_stress_pnorm_matches_oracle(ctx, hx, orc):
    dims = (11, 6, 5)
    nodes, el, c0 = _setup(ctx, hx, dims)
    rng = np.random.default_rng(21)
    u = rng.standard_normal(3 * nodes.shape[0]) * 1e-2
    dens = rng.uniform(0, 1, c0.shape[0])
    dens[::5] = 1e-8  # void elements contribute nothing
    for P in (1.0, 8.0, 32.0):
        pn, vmax = ctx.stress_pnorm(u, dens, 1.5, 0.3, P)
        want, wmax = orc.stress_pnorm(c0, nodes, u, 1.5, 0.3, dens, P)
        assert vmax == pytest.approx(wmax, rel=1e-12)
        assert pn == pytest.approx(want, rel=1e-12)
    # the aggregate lies between the max and N^(1/P) times the max
    pn8, vmax = ctx.stress_pnorm(u, dens, 1.5, 0.3, 8.0)
    assert vmax <= pn8 <= vmax * c0.shape[0] ** (1 / 8.0)


def test_compute_stress_field_reference_shaped(ctx, hx, orc):
    from importlib import import_module
    api = import_module("2025_12_09_hexat_v069_b200.api")
    dims = (6, 5, 4)
    nodes, el, _ = hx.mesh.generate_mesh(*dims)
    c0 = hx.mesh.connectivity0(el)
    rng = np.random.default_rng(13)
    u = (rng.standard_normal(3 * nodes.shape[0]) * 1e-2).astype(np.float32)
    dens = rng.uniform(0, 1, c0.shape[0]).astype(np.float32)
    pr, vm, vo, l1, dr = api.compute_stress_field(nodes, el, u, 1.0, 0.3, dens, ctx=ctx)
    want = orc.stress(c0, nodes, u, 1.0 * 1.0, 0.3, dens)
    assert pr.shape == (3, c0.shape[0]) and vo.shape == (6, c0.shape[0])
    assert np.abs(vm - want[1]).max() <= 1e-5 * np.abs(want[1]).max()
    assert np.abs(pr.T - want[0]).max() <= 1e-5 * np.abs(want[0]).max()


def test_energy_compliance_oc(ctx, hx, orc):
    dims = (14, 6, 5)
    nodes, el, c0 = _setup(ctx, hx, dims)
    rng = np.random.default_rng(14)
    u = rng.standard_normal(3 * nodes.shape[0])
    f = rng.standard_normal(3 * nodes.shape[0])
    ce = ctx.element_energy(u, c0.shape[0])
    assert np.abs(ce - orc.element_energy(c0, orc.canonical_ke(), u)).max() <= 1e-12 * ce.max()
    assert ctx.compliance(f, u) == pytest.approx(np.dot(f, u), rel=1e-12)
    x = rng.uniform(0.2, 0.45, c0.shape[0])
    dc = -rng.uniform(0.1, 2.0, c0.shape[0])
    dv = np.ones_like(x)
    xn, lam, steps = ctx.oc_update(x, dc, dv, 0.3, 0.2)
    xo, lamo, stepso = orc.oc_update(x, dc, dv, 0.3, 0.2)
    assert steps == stepso and lam == pytest.approx(lamo, rel=1e-12)
    assert np.abs(xn - xo).max() <= 1e-14


def test_solve_system_gpu_unpruned(ctx, hx, orc):
    from importlib import import_module
    api = import_module("2025_12_09_hexat_v069_b200.api")
    dims = (12, 4, 4)
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    dens = np.random.default_rng(15).uniform(0.2, 1.0, el.shape[0]).astype(np.float32)
    E = 2.5
    x, rel, name = api.solve_system_gpu(nodes, el, E, 0.3, bc, f.astype(np.float32), dens,
                                        tol=1e-6, shift_factor=1e-7, ctx=ctx)
    assert name == "Jacobi" and rel < 1e-6 and x.dtype == np.float32
    c0 = hx.mesh.connectivity0(el)
    ke = orc.canonical_ke()
    fac = E * dens.astype(np.float64)
    nN = nodes.shape[0]
    free = orc.free_mask_from(bc, orc.diagonal(c0, nN, ke, fac))
    uo, _, _, _ = orc.cg_solve(c0, nN, ke, fac, free, f.astype(np.float32) * free, tol=1e-10,
                               shift_factor=np.float32(1e-7), precond_add=True)
    assert np.abs(x - uo).max() <= 2e-5 * np.abs(uo).max()


def test_solve_system_gpu_pruned_mesh(ctx, hx, orc):
    """The reference prunes void elements and renumbers before its GPU solve
    (src/Solvers/Solver.jl:60-91): the pruned, renumbered mesh goes through
    the lattice embedding and must give the reference's reconstructed u."""
    from importlib import import_module
    api = import_module("2025_12_09_hexat_v069_b200.api")
    dims = (14, 6, 5)
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    rng = np.random.default_rng(16)
    dens = rng.uniform(0.3, 1.0, el.shape[0]).astype(np.float32)
    cent = np.stack([(np.arange(el.shape[0]) % dims[0])], 1)
    hole = (cent[:, 0] > 4) & (cent[:, 0] < 9) & (rng.uniform(size=el.shape[0]) < 0.7)
    dens[hole] = 1e-3
    thr = np.float32(1e-3) * np.float32(1.01)
    pn, pe, pbc, pf, pd, n2o = prune_system(nodes, el, dens, thr, bc, f.astype(np.float32))
    x, rel, name = api.solve_system_gpu(pn, pe, 1.0, 0.3, pbc, pf, pd, tol=1e-7,
                                        shift_factor=0.0, min_stiffness_threshold=1e-3, ctx=ctx)
    u_full = reconstruct_full_solution(x, n2o, nodes.shape[0])
    # oracle on the pruned (renumbered) mesh
    c0 = hx.mesh.connectivity0(pe)
    ke = orc.canonical_ke()
    fac = pd.astype(np.float64)
    free = orc.free_mask_from(pbc, orc.diagonal(c0, pn.shape[0], ke, fac))
    uo, _, _, _ = orc.cg_solve(c0, pn.shape[0], ke, fac, free, pf * free, tol=1e-10)
    uo_full = reconstruct_full_solution(uo, n2o, nodes.shape[0])
    assert rel < 1e-7
    assert np.abs(u_full - uo_full).max() <= 2e-5 * np.abs(uo_full).max()


def test_solve_system_grid_device_pruning_matches_pruned_path(ctx, hx, orc):
    """The unpruned grid plus min_stiffness_threshold, pruned on the device
    (hx_solve_system_grid), against the reference's host path: prune_system
    (src/Mesh/MeshPruner.jl:18-112), the solve on the pruned, renumbered mesh
    (hx_solve_system_gpu, lattice embedding) and reconstruct_full_solution;
    and both against the oracle's solve of the pruned mesh."""
    from importlib import import_module
    api = import_module("2025_12_09_hexat_v069_b200.api")
    dims = (14, 6, 5)
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    rng = np.random.default_rng(17)
    dens = rng.uniform(0.3, 1.0, el.shape[0]).astype(np.float32)
    i = np.arange(el.shape[0]) % dims[0]
    hole = (i > 4) & (i < 9) & (rng.uniform(size=el.shape[0]) < 0.7)
    dens[hole] = 1e-3
    thr = np.float32(1e-3) * np.float32(1.01)
    f32 = f.astype(np.float32)
    xg, relg, name = api.solve_system_grid(dims, (1.0, 1.0, 1.0), 1.0, 0.3, bc, f32, dens,
                                           tol=1e-7, shift_factor=0.0,
                                           min_stiffness_threshold=thr, ctx=ctx)
    assert name == "Jacobi" and relg < 1e-7
    pn, pe, pbc, pf, pd, n2o = prune_system(nodes, el, dens, thr, bc, f32)
    xp, relp, _ = api.solve_system_gpu(pn, pe, 1.0, 0.3, pbc, pf, pd, tol=1e-7,
                                       shift_factor=0.0, min_stiffness_threshold=thr, ctx=ctx)
    up = reconstruct_full_solution(xp, n2o, nodes.shape[0])
    assert np.abs(xg - up).max() <= 1e-5 * np.abs(up).max()
    # nodes outside the pruned mesh are exactly zero, as reconstruct returns
    gone = np.ones(nodes.shape[0], bool)
    gone[n2o] = False
    assert np.all(xg.reshape(-1, 3)[gone] == 0)
    c0 = hx.mesh.connectivity0(pe)
    fac = pd.astype(np.float64)
    free = orc.free_mask_from(pbc, orc.diagonal(c0, pn.shape[0], orc.canonical_ke(), fac))
    uo, _, _, _ = orc.cg_solve(c0, pn.shape[0], orc.canonical_ke(), fac, free, pf * free,
                               tol=1e-10)
    uo_full = reconstruct_full_solution(uo, n2o, nodes.shape[0])
    assert np.abs(xg - uo_full).max() <= 2e-5 * np.abs(uo_full).max()
