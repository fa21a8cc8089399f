"""The learned preconditioner
P = D^-1/2 (I + sum_l R_l^T E_l^T G_l^T G_l E_l R_l) D^-1/2  (levels L0..L0+2):
the BF16 tensor-core convolutions of G and G^T and the weight gradient, and
the whole application of P, checked against a CPU reference built on torch
(FP32 arithmetic with the kernels' BF16 roundings of weights, activations
and gradients); P symmetric positive definite; training on solver-generated
residual/error pairs; flexible CG with the trained networks against plain
Jacobi-PCG; the fallback path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LP = 27 * 256
NP = 4 * LP       # one network
NETS = 3          # networks on node-grid levels L0 .. L0 + 2
L0 = 2            # HX_NET_FIRST_LEVEL
NET_IN = 6


def _bf(a):
    import torch
    return a.to(torch.bfloat16).to(torch.float32)


def _weights(params, k):
    """BF16-rounded conv weights of network k as torch [co][ci][kz][ky][kx]."""
    import torch
    return [_bf(torch.from_numpy(params[k * NP + l * LP:k * NP + (l + 1) * LP].reshape(27, 16, 16))
                .permute(1, 2, 0).reshape(16, 16, 3, 3, 3)) for l in range(4)]


def _gtg(W, x):
    """G^T G x with BF16 rounding of every layer output (x: [1, 16, z, y, x])."""
    import torch.nn.functional as F
    a = [x]
    for l in range(4):
        a.append(_bf(F.conv3d(a[-1], W[l], padding=1)))
    b = {4: a[4]}
    for l in (3, 2, 1, 0):
        b[l] = _bf(F.conv_transpose3d(b[l + 1], W[l], padding=1))
    return a, b


def _torch_reference(params, dims, x0, dy):
    """y = G^T G x0 and d<dy, y>/dW for network 0 in torch (CPU, FP32),
    rounding to BF16 where the GPU kernels store BF16: every layer output,
    forward and backward."""
    import torch
    import torch.nn.functional as F
    nx, ny, nz = dims

    def vol(a):  # [node][16] (x fastest) -> [1, 16, z, y, x]
        return torch.from_numpy(a.reshape(nz, ny, nx, 16)).permute(3, 0, 1, 2)[None].float()

    def unvol(t):
        return t[0].permute(1, 2, 3, 0).reshape(-1, 16).numpy()

    W = _weights(params, 0)
    conv = lambda x, l: _bf(F.conv3d(x, W[l], padding=1))
    convT = lambda x, l: _bf(F.conv_transpose3d(x, W[l], padding=1))
    wgrad = lambda X, D: torch.nn.grad.conv3d_weight(X, W[0].shape, D, padding=1)
    a, b = _gtg(W, _bf(vol(x0)))
    gw = [torch.zeros_like(W[0]) for _ in range(4)]
    e = _bf(vol(dy))
    for l in range(4):                    # transposed uses: X = dLoss/dout, D = input
        gw[l] += wgrad(e, b[l + 1])
        e = conv(e, l)
    for l in (3, 2, 1, 0):                # forward uses: X = input, D = dLoss/dout
        gw[l] += wgrad(a[l], e)
        if l > 0:
            e = convT(e, l)
    grads = np.concatenate([g.reshape(16, 16, 27).permute(2, 0, 1).reshape(-1).numpy()
                            for g in gw])
    return unvol(b[0]), grads


def test_conv_stack_and_gradient_match_torch(ctx):
    dims = (21, 11, 6)  # several 16x8x4 tiles, partial at every edge
    nn_ = dims[0] * dims[1] * dims[2]
    rng = np.random.default_rng(7)
    ctx.net_init(seed=11)
    p = ctx.net_get_params()
    p = (p + rng.normal(0, 0.02, p.size).astype(np.float32))
    ctx.net_set_params(p)
    p = ctx.net_get_params()  # unused input channels forced to zero
    assert not p.reshape(NETS, 4, 27, 16, 16)[:, 0, :, :, NET_IN:].any()
    x0 = np.zeros((nn_, 16), np.float32)
    x0[:, :NET_IN] = rng.standard_normal((nn_, NET_IN))
    dy = np.zeros((nn_, 16), np.float32)
    dy[:, :NET_IN] = rng.standard_normal((nn_, NET_IN))
    y, g = ctx.net_forward_backward(dims, x0, dy)
    yr, gr = _torch_reference(p, dims, x0, dy)
    assert not y[:, NET_IN:].any()
    assert np.abs(y - yr).max() <= 2e-2 * np.abs(yr).max()
    assert np.abs(y - yr).mean() <= 2e-3 * np.abs(yr).max()
    for l in range(4):
        a, b = g[l * LP:(l + 1) * LP], gr[l * LP:(l + 1) * LP]
        assert np.abs(a - b).max() <= 3e-2 * np.abs(b).max(), l
        assert np.abs(a - b).mean() <= 3e-3 * np.abs(b).max(), l
    assert np.isfinite(g).all() and not g[NP:].any()


def _problem(ctx, hx, dims, seed):
    import torch
    W = hx.workloads
    nodes, el, bc, f = W.cantilever(*dims)
    ctx.set_grid(*dims)
    ctx.set_material(1.0, 0.3)
    ctx.set_bc(bc)
    raw = W.raw_density(el.shape[0], seed)
    rho_f, _ = ctx.filter(raw, 2.0, 0, 1e-5, 200)
    fac = W.simp(W.map_density(rho_f, 1e-3))
    dev = torch.device("cuda", 0)
    return torch.from_numpy(f).to(dev), torch.from_numpy(fac).to(dev)


def _restrict(x, normalise=False):
    """Full weighting (1/2, 1, 1/2 per axis) onto the next coarser node grid."""
    import torch
    import torch.nn.functional as F
    w1 = torch.tensor([0.5, 1.0, 0.5])
    k = (w1[:, None, None] * w1[None, :, None] * w1[None, None, :])[None, None]
    C = x.shape[1]
    out = F.conv3d(x, k.expand(C, 1, 3, 3, 3).to(x.dtype), stride=2, padding=1, groups=C)
    if normalise:
        out = out / F.conv3d(torch.ones_like(x[:, :1]), k.to(x.dtype), stride=2, padding=1)
    return out


def _prolong(x, fine_shape):
    """Exact transpose of _restrict (no normalisation)."""
    import torch
    import torch.nn.functional as F
    w1 = torch.tensor([0.5, 1.0, 0.5])
    k = (w1[:, None, None] * w1[None, :, None] * w1[None, None, :])[None, None]
    C = x.shape[1]
    op = tuple(fine_shape[i] - 2 * x.shape[2 + i] + 1 for i in range(3))
    return F.conv_transpose3d(x, k.expand(C, 1, 3, 3, 3).to(x.dtype), stride=2, padding=1,
                              output_padding=op, groups=C)


def _torch_precond(params, dims, fac, minv, r):
    """P r restated in torch from the preconditioner's definition."""
    import torch
    nx, ny, nz = dims
    nz1, ny1, nx1 = nz + 1, ny + 1, nx + 1
    dinvs = np.sqrt(minv)
    n = r.size
    s = np.sqrt(float(r @ (minv * r)) / n)
    x = torch.from_numpy((dinvs * r / s).astype(np.float32)).reshape(nz1, ny1, nx1, 3)
    x = x.permute(3, 0, 1, 2)[None]
    # nodal density feature: mean over the node's elements of clip((log10 f + 9) / 9)
    v = np.clip((np.log10(np.maximum(fac, 1e-12)) + 9.0) / 9.0, 0.0, 1.0).reshape(nz, ny, nx)
    vp = np.pad(v, 1)
    cp = np.pad(np.ones_like(v), 1)
    ssum = sum(vp[a:a + nz1, b:b + ny1, c:c + nx1] for a in (0, 1) for b in (0, 1) for c in (0, 1))
    cnt = sum(cp[a:a + nz1, b:b + ny1, c:c + nx1] for a in (0, 1) for b in (0, 1) for c in (0, 1))
    feat = [torch.from_numpy((ssum / cnt).astype(np.float32))[None, None]]
    xs = [x]
    top = L0 + NETS - 1
    for l in range(1, top + 1):
        feat.append(_restrict(feat[-1], True))
        xs.append(_restrict(xs[-1]))
    acc = None
    for l in range(top, 0, -1):
        if l >= L0:
            X0 = torch.zeros((1, 16) + xs[l].shape[2:])
            X0[:, :3] = _bf(xs[l])
            X0[:, 3:6] = _bf(xs[l] * feat[l])
            _, b = _gtg(_weights(params, l - L0), X0)
            t = b[0][:, :3] + feat[l] * b[0][:, 3:6]
            acc = t if acc is None else t + _prolong(acc, xs[l].shape[2:])
        else:
            acc = _prolong(acc, xs[l].shape[2:])
    acc = _prolong(acc, xs[0].shape[2:])
    corr = acc[0].permute(1, 2, 3, 0).reshape(-1).double().numpy()
    return minv * r + s * dinvs * corr, minv * r


def test_full_preconditioner_matches_torch(ctx, hx):
    import torch
    dims = (30, 13, 11)  # odd and even node counts on the levels
    f_d, fac_d = _problem(ctx, hx, dims, seed=6)
    ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), torch.zeros_like(f_d).data_ptr(),
                     opts=hx.default_opts(tol=1e-2))
    ctx.net_init(seed=21)
    p = ctx.net_get_params()
    rng = np.random.default_rng(2)
    ctx.net_set_params(p * 2.0 + rng.normal(0, 0.01, p.size).astype(np.float32))
    p = ctx.net_get_params()
    ctx.net_prepare(fac_d.data_ptr())
    fac = fac_d.cpu().numpy()
    bc = hx.workloads.cantilever(*dims, with_elements=False)[2].reshape(-1)
    diag = ctx.diagonal(fac, f_d.numel())
    minv = np.where(bc > 0, 0.0, 1.0 / diag)
    r = rng.standard_normal(f_d.numel()) * (bc == 0)
    z = torch.empty_like(f_d)
    ctx.net_apply(torch.from_numpy(r).to(f_d.device).data_ptr(), z.data_ptr())
    z = z.cpu().numpy()
    zr, jac = _torch_precond(p, dims, fac, minv, r)
    corr = np.linalg.norm(zr - jac)
    assert corr > 0.1 * np.linalg.norm(jac)  # the networks contribute
    assert np.linalg.norm(z - zr) <= 2e-2 * corr
    assert np.array_equal(z[bc > 0], np.zeros(int((bc > 0).sum())))


def test_preconditioner_is_symmetric_positive_definite(ctx, hx):
    import torch
    dims = (24, 8, 8)
    f_d, fac_d = _problem(ctx, hx, dims, seed=4)
    ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), torch.zeros_like(f_d).data_ptr(),
                     opts=hx.default_opts(tol=1e-3))
    ctx.net_init(seed=3)
    p = ctx.net_get_params()
    ctx.net_set_params(p * 3.0)  # a strong correction, far from Jacobi
    ctx.net_prepare(fac_d.data_ptr())
    g = torch.Generator(device="cpu").manual_seed(1)
    bc = hx.workloads.cantilever(*dims, with_elements=False)[2]
    free = torch.from_numpy(bc.reshape(-1) == 0).to(f_d.device)
    r = [torch.randn(f_d.numel(), generator=g, dtype=torch.float64).to(f_d.device) * free
         for _ in range(3)]
    z = []
    for v in r:
        out = torch.empty_like(v)
        ctx.net_apply(v.data_ptr(), out.data_ptr())
        z.append(out)
    for i in range(3):
        assert float(r[i] @ z[i]) > 0
        for j in range(i):
            a, b = float(r[i] @ z[j]), float(r[j] @ z[i])
            scale = np.sqrt(float(r[i] @ z[i]) * float(r[j] @ z[j]))
            assert abs(a - b) <= 1e-2 * scale, (i, j, a, b)
    # linearity in r (up to the BF16 roundings): P(2 r0 + r1) = 2 P r0 + P r1
    out = torch.empty_like(r[0])
    ctx.net_apply((2 * r[0] + r[1]).data_ptr(), out.data_ptr())
    ref = 2 * z[0] + z[1]
    assert float(torch.linalg.norm(out - ref) / torch.linalg.norm(ref)) < 2e-2
    # zero residual -> zero
    zero = torch.zeros_like(r[0])
    ctx.net_apply(zero.data_ptr(), out.data_ptr())
    assert not out.any()


def test_training_reduces_loss_and_iterations(ctx, hx):
    """Training from a fresh initialisation on one problem's Jacobi-PCG
    snapshots (mini-batches of 4): the loss falls and flexible CG with the
    trained networks converges on the true residual in at least 1.5x fewer
    iterations than Jacobi-PCG."""
    import torch
    dims = (64, 24, 24)  # coarse network levels of some extent (17x7x7 .. 5x2x2)
    f_d, fac_d = _problem(ctx, hx, dims, seed=3)
    n = f_d.numel()
    # reference solution and Jacobi-PCG snapshots
    u_star = torch.zeros_like(f_d)
    ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u_star.data_ptr(),
                     opts=hx.default_opts(tol=1e-11, max_iter=100000))
    base_iters = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(),
                                  torch.zeros_like(f_d).data_ptr(),
                                  opts=hx.default_opts(tol=1e-6)).iterations
    snaps = torch.zeros((64, n), dtype=torch.float64, device=f_d.device)
    taken = ctx.pcg_snapshots(f_d.data_ptr(), fac_d.data_ptr(), 8, 64, 1e-8, snaps.data_ptr())
    assert taken >= 8
    ctx.net_init(seed=5)
    ctx.net_prepare(fac_d.data_ptr())
    B = 4
    R = torch.empty((B, n), dtype=torch.float64, device=f_d.device)
    E = torch.empty_like(R)
    losses = []
    rng = np.random.default_rng(0)
    for step in range(500):
        for b, k in enumerate(rng.integers(taken, size=B)):
            ctx.residual_device(f_d.data_ptr(), fac_d.data_ptr(), snaps[k].data_ptr(),
                                R[b].data_ptr())
            torch.sub(u_star, snaps[k], out=E[b])
        torch.cuda.current_stream().synchronize()
        losses.append(ctx.net_train_batch([R[b].data_ptr() for b in range(B)],
                                          [E[b].data_ptr() for b in range(B)],
                                          3e-4 if step < 250 else 1e-4))
    first = np.mean(losses[:50])
    last = np.mean(losses[-50:])
    assert np.isfinite(losses).all() and last < first
    # flexible CG with the trained networks: converges on the true residual
    u = torch.zeros_like(f_d)
    rl = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u.data_ptr(),
                          opts=hx.default_opts(tol=1e-6, preconditioner=1, max_iter=20000,
                                               learned_no_fallback=1))
    assert rl.status == 0 and rl.true_rel_res < 1e-6
    err = float(torch.linalg.norm(u - u_star) / torch.linalg.norm(u_star))
    assert err < 1e-4
    print(f"jacobi-pcg {base_iters} its; learned fcg {rl.iterations} its; "
          f"loss {first:.3e} -> {last:.3e}")
    # the gain: at least 1.5x fewer iterations than Jacobi-PCG
    assert rl.iterations * 1.5 < base_iters


def test_poisoned_network_falls_back_to_jacobi(ctx, hx):
    import torch
    dims = (24, 8, 8)
    f_d, fac_d = _problem(ctx, hx, dims, seed=9)
    ctx.net_init(seed=1)
    p = ctx.net_get_params()
    p[:] = 1e30  # the network now outputs inf/NaN
    ctx.net_set_params(p)
    u = torch.zeros_like(f_d)
    rl = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u.data_ptr(),
                          opts=hx.default_opts(tol=1e-6, preconditioner=1, max_iter=20000))
    assert rl.fallback_used == 1
    assert rl.status == 0 and rl.true_rel_res < 1e-6


def test_batch_step_sums_single_gradients(ctx, hx):
    """A batch of two copies of one pair: the same loss as the single step,
    and an Adam step along the same direction.  The first Adam step moves a
    parameter by -lr g / (|g| + eps); for the summed gradient 2g this differs
    by at most lr eps / (2 |g|), i.e. < 0.01 lr where |g| > 99 eps, which is
    where the single step moved it by more than 0.99 lr."""
    import torch
    dims = (20, 8, 6)
    f_d, fac_d = _problem(ctx, hx, dims, seed=12)
    x = torch.zeros_like(f_d)
    ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), x.data_ptr(),
                     opts=hx.default_opts(tol=1e-2))
    u_star = torch.zeros_like(f_d)
    ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u_star.data_ptr(),
                     opts=hx.default_opts(tol=1e-10, max_iter=100000))
    r = torch.empty_like(f_d)
    ctx.residual_device(f_d.data_ptr(), fac_d.data_ptr(), x.data_ptr(), r.data_ptr())
    e = (u_star - x).contiguous()
    lr = 1e-3
    ctx.net_init(seed=4)
    p0 = ctx.net_get_params()
    ctx.net_prepare(fac_d.data_ptr())
    l1 = ctx.net_train_step(r.data_ptr(), e.data_ptr(), lr)
    d1 = ctx.net_get_params() - p0
    ctx.net_init(seed=4)
    l2 = ctx.net_train_batch([r.data_ptr(), r.data_ptr()], [e.data_ptr(), e.data_ptr()], lr)
    d2 = ctx.net_get_params() - p0
    assert l1 == l2
    big = np.abs(d1) > 0.99 * lr
    assert big.sum() > 1000
    assert np.abs(d1 - d2)[big].max() <= 0.01 * lr
    assert np.array_equal(np.sign(d1[big]), np.sign(d2[big]))


def test_shipped_weights_gain_on_unseen_problem(ctx, hx):
    """The committed networks (trained on a mixture of grids up to 128x64x64)
    on an unseen seeded problem: FCG converges on the true residual in at
    least 1.6x fewer iterations than Jacobi-PCG (the gain grows with the
    grid: 5.3x at 320x160x160)."""
    import torch
    from importlib import import_module
    learned = import_module(hx.__name__ + ".learned")
    f_d, fac_d = learned.problem(ctx, (96, 48, 48), seed=77)
    rj = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), torch.zeros_like(f_d).data_ptr(),
                          opts=hx.default_opts(tol=1e-6, max_iter=100000))
    learned.load_into(ctx)
    u = torch.zeros_like(f_d)
    rl = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u.data_ptr(),
                          opts=hx.default_opts(tol=1e-6, preconditioner=1, max_iter=100000))
    print(f"96x48x48: jacobi-pcg {rj.iterations} its; learned fcg {rl.iterations} its "
          f"(fallback {rl.fallback_used})")
    assert rl.status == 0 and rl.true_rel_res < 1e-6 and rl.fallback_used == 0
    assert rl.iterations * 1.6 < rj.iterations


def test_mixed_precision_learned_fcg(ctx, hx):
    """FP32 flexible CG with the committed networks inside FP64 reliable
    updates: converges on the FP64 true residual without fallback, in
    fewer iterations than FP64 Jacobi-PCG, to the FP64 solution."""
    import torch
    from importlib import import_module
    learned = import_module(hx.__name__ + ".learned")
    f_d, fac_d = learned.problem(ctx, (96, 48, 48), seed=78)
    u64 = torch.zeros_like(f_d)
    rj = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u64.data_ptr(),
                          opts=hx.default_opts(tol=1e-6, max_iter=100000))
    learned.load_into(ctx)
    u = torch.zeros_like(f_d)
    rl = ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), u.data_ptr(),
                          opts=hx.default_opts(tol=1e-6, preconditioner=1, precision=1,
                                               max_iter=100000))
    print(f"96x48x48 mixed: jacobi-pcg fp64 {rj.iterations} its; learned fcg fp32 "
          f"{rl.iterations} its, {rl.refinements} residual replacements")
    assert rl.status == 0 and rl.true_rel_res < 1e-6 and rl.fallback_used == 0
    assert rl.iterations * 1.5 < rj.iterations
    err = float(torch.linalg.norm(u - u64) / torch.linalg.norm(u64))
    assert err < 1e-4
    c64, c = float(f_d @ u64), float(f_d @ u)
    assert abs(c - c64) <= 1e-5 * abs(c64)


def test_conv_wait_timeout_is_reported(ctx, hx):
    """Failure detection without a fault: a convolution CTA whose barrier is
    never armed gives up after its bounded wait, the host reads the error,
    and the context keeps working (the preconditioner gives the same result
    as before the test, so the weights were restored)."""
    import time
    import torch
    dims = (24, 8, 8)
    f_d, fac_d = _problem(ctx, hx, dims, seed=5)
    ctx.solve_device(f_d.data_ptr(), fac_d.data_ptr(), torch.zeros_like(f_d).data_ptr(),
                     opts=hx.default_opts(tol=1e-3))
    ctx.net_init(seed=8)
    ctx.net_prepare(fac_d.data_ptr())
    z0, z1 = torch.empty_like(f_d), torch.empty_like(f_d)
    ctx.net_apply(f_d.data_ptr(), z0.data_ptr())
    t0 = time.time()
    assert ctx.selftest_wait_timeout()
    assert time.time() - t0 < 30.0
    ctx.net_apply(f_d.data_ptr(), z1.data_ptr())
    assert torch.equal(z0, z1)
