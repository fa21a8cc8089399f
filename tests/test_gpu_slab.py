"""The slab-decomposed solve's device path (slab.py with the library's
operator per slab, DeviceSlabOperator) on one GPU: a one-rank NCCL group
(no exchange partner) must reproduce the library's own FP64 Jacobi-PCG
solve.  The exchange and the owner-weighted reductions are covered with two
and three gloo ranks on CPU (tests/test_slab.py); several GPUs are not
available to these tests."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_one_rank_device_slab_matches_library_solve(ctx, hx, orc):
    import torch
    import torch.distributed as dist
    from importlib import import_module
    slab_mod = import_module(hx.__name__ + ".slab")
    dims = (20, 8, 10)
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    fac = hx.workloads.simp(np.random.default_rng(3).uniform(0.2, 1.0, el.shape[0]))
    ctx.set_grid(*dims)
    ctx.set_material(1.0, 0.3)
    ctx.set_bc(bc)
    u_lib, rep = ctx.solve(f, fac, tol=1e-10)
    store = dist.HashStore()
    dist.init_process_group("nccl", store=store, rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        S = slab_mod.Slab(dims, 0, 1)
        dev = torch.device("cuda", 0)
        fac_d = torch.from_numpy(fac).to(dev)
        op = slab_mod.DeviceSlabOperator(S, fac_d)
        c0 = hx.mesh.connectivity0(el)
        diag = torch.from_numpy(orc.diagonal(c0, nodes.shape[0], orc.canonical_ke(), fac)).to(dev)
        free = torch.from_numpy((~(np.asarray(bc) > 0)).reshape(-1).astype(np.float64)).to(dev)
        b = torch.from_numpy(f).to(dev)
        u, it, rel, _ = slab_mod.pcg(S, dist, op, diag, free, b, tol=1e-10)
        u = u.cpu().numpy()
    finally:
        dist.destroy_process_group()
    assert rel < 1e-10 and abs(it - rep.iterations) <= 2
    assert np.abs(u - u_lib).max() <= 1e-8 * np.abs(u_lib).max()
