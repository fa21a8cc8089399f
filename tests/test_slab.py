"""(CPU, gloo) The slab decomposition of the multi-GPU solve (slab.py): two
and three ranks on CPU, each applying the ORACLE's element-by-element K.u
(the restatement of CPUSolver.apply_stiffness) to its slab of element
planes, exchanging the shared node planes and all-reducing the dot products
through torch.distributed (gloo).  The partitioned operator must equal the
single-domain oracle product to 1e-13, and the partitioned Jacobi-PCG the
single-domain oracle solve (hxo_cg_solve, the same algorithm and stopping
rule) to 1e-12, with the same iteration count."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _problem(dims):
    import importlib
    hx = importlib.import_module("2025_12_09_hexat_v069_b200")
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    rng = np.random.default_rng(4)
    fac = hx.workloads.simp(rng.uniform(0.4, 1.0, el.shape[0]))
    free = (~(np.asarray(bc) > 0)).reshape(-1).astype(np.float64)
    return f, fac, free


def _rank(rank, world, port, dims, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import importlib
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        slab_mod = importlib.import_module("2025_12_09_hexat_v069_b200.slab")
        from oracle import oracle
        f, fac, free = _problem(dims)
        S = slab_mod.Slab(dims, rank, world)
        conn = oracle.structured_conn0(dims[0], dims[1], S.nzl)
        nn_l = S.n // 3
        ke = oracle.canonical_ke()
        fac_l = fac[S.elem_slice()]

        def apply_local(x):
            return torch.from_numpy(oracle.apply_stiffness(conn, nn_l, ke, fac_l, x.numpy(),
                                                           nthreads=1))

        # the partitioned operator on a random vector
        rng = np.random.default_rng(11)
        xg = rng.standard_normal(f.shape[0])
        y = slab_mod.halo_sum(apply_local(torch.from_numpy(xg[S.node_slice()].copy())), S, dist)
        yg = slab_mod.gather(y, S, dist).numpy()
        diag_l = torch.from_numpy(oracle.diagonal(conn, nn_l, ke, fac_l))
        b = torch.from_numpy((f * free)[S.node_slice()].copy())
        u, it, rel, _ = slab_mod.pcg(S, dist, apply_local, diag_l,
                                     torch.from_numpy(free[S.node_slice()].copy()), b,
                                     tol=1e-13, max_iter=5000)
        ug = slab_mod.gather(u, S, dist).numpy()
        if rank == 0:
            q.put(("ok", yg, ug, it, rel))
    except Exception as e:  # reported to the parent; every rank leaves the group
        q.put(("error", repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,dims", [(2, (6, 3, 8)), (3, (5, 3, 7))])
def test_slab_pcg_matches_single_domain_oracle(orc, world, dims):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, dims, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        res = q.get(timeout=300)
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.kill()
    assert res[0] == "ok", res
    _, yg, ug, it, rel = res
    f, fac, free = _problem(dims)
    import importlib
    hx = importlib.import_module("2025_12_09_hexat_v069_b200")
    _, el, _ = hx.mesh.generate_mesh(*dims)
    c0 = hx.mesh.connectivity0(el)
    nn = f.shape[0] // 3
    ke = orc.canonical_ke()
    rng = np.random.default_rng(11)
    xg = rng.standard_normal(f.shape[0])
    y1 = orc.apply_stiffness(c0, nn, ke, fac, xg)
    assert np.abs(yg - y1).max() <= 1e-13 * np.abs(y1).max()
    fm = orc.free_mask_from(free == 0, orc.diagonal(c0, nn, ke, fac))
    uo, ito, relo, _ = orc.cg_solve(c0, nn, ke, fac, fm, f * fm, tol=1e-13, max_iter=5000)
    assert it == ito and rel < 1e-13
    assert np.abs(ug - uo).max() <= 1e-12 * np.abs(uo).max()
    assert np.all(ug[fm == 0] == 0)


def test_split_planes():
    import importlib
    slab_mod = importlib.import_module("2025_12_09_hexat_v069_b200.slab")
    assert slab_mod.split_planes(7, 3) == [(0, 3), (3, 5), (5, 7)]
    assert slab_mod.split_planes(160, 8)[-1] == (140, 160)
    with pytest.raises(ValueError):
        slab_mod.split_planes(2, 3)
    s = slab_mod.Slab((320, 160, 160), 1, 4)
    assert s.n == 3 * 321 * 161 * 41 and s.owned() == slice(0, s.n - 3 * 321 * 161)
