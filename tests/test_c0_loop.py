"""The C0 topology-optimisation loop (cantilever 60x20x20, 50 OC iterations)
against the golden fixture that the CPU oracle produced
(tests/golden/make_c0_golden.py): the fixture's own consistency on the CPU,
and the GPU library's loop (filter, warm-started solves, energies, OC
update) on the GPU."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c0_oc_loop.npz")


def _golden():
    g = np.load(GOLDEN)
    params = {k: g[k].item() for k in ("volfrac", "radius", "n_iter", "p", "e0", "emin", "nu",
                                       "move", "tol", "ref_compat", "filter_tol",
                                       "filter_max_iter")}
    return g, params


def test_golden_fixture_is_consistent(hx, orc):
    g, prm = _golden()
    dims = tuple(int(v) for v in g["dims"])
    hist, x = g["compliance"], g["x"]
    assert hist.shape == (prm["n_iter"],) and np.isfinite(hist).all()
    assert hist[-1] < 0.2 * hist[0]                       # the design stiffened
    assert x.mean() <= prm["volfrac"] * (1 + 1e-9)        # volume constraint
    assert x.min() >= 0.0 and x.max() <= 1.0
    # the oracle reproduces the start of the history (thread-count rounding only)
    W = hx.workloads
    nodes, el, bc, f = W.cantilever(*dims)
    conn0 = hx.mesh.connectivity0(el)
    p3 = dict(prm, n_iter=3)
    h3, _, _ = orc.topopt_oc_loop(conn0, nodes.shape[0], dims, bc, f, **p3)
    assert np.allclose(h3, hist[:3], rtol=1e-9, atol=0)


@pytest.mark.gpu
def test_gpu_oc_loop_matches_oracle(ctx, hx):
    from importlib import import_module
    topopt = import_module(hx.__name__ + ".topopt")
    g, prm = _golden()
    dims = tuple(int(v) for v in g["dims"])
    W = hx.workloads
    nodes, el, bc, f = W.cantilever(*dims)
    ctx.set_grid(*dims)
    res = topopt.run_oc(ctx, bc, f, prm["volfrac"], prm["radius"], prm["n_iter"], p=prm["p"],
                        e0=prm["e0"], emin=prm["emin"], nu=prm["nu"], move=prm["move"],
                        tol=prm["tol"], ref_compat=prm["ref_compat"],
                        filter_tol=prm["filter_tol"], filter_max_iter=prm["filter_max_iter"])
    c = np.array(res.compliance)
    rel = np.abs(c - g["compliance"]) / g["compliance"]
    print(f"C0 loop: compliance {c[0]:.6g} -> {c[-1]:.6g}; max rel diff to the oracle "
          f"{rel.max():.2e}; final rho max abs diff {np.abs(res.rho - g['rho']).max():.2e}")
    # both sides solve to rtol 1e-6, so the loops agree to that order
    assert rel[0] <= 1e-6
    assert rel.max() <= 1e-4
    assert np.abs(res.rho - g["rho"]).max() <= 1e-3
    assert np.abs(res.x - g["x"]).max() <= 1e-3


@pytest.mark.gpu
def test_gpu_device_loop_matches_oracle(ctx, hx):
    """The device-resident loop (all pieces on the GPU) against the fixture."""
    from importlib import import_module
    topopt = import_module(hx.__name__ + ".topopt")
    g, prm = _golden()
    dims = tuple(int(v) for v in g["dims"])
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    ctx.set_grid(*dims)
    res = topopt.run_oc_device(ctx, bc, f, prm["volfrac"], prm["radius"], prm["n_iter"],
                               p=prm["p"], e0=prm["e0"], emin=prm["emin"], nu=prm["nu"],
                               move=prm["move"], tol=prm["tol"], ref_compat=prm["ref_compat"],
                               filter_tol=prm["filter_tol"],
                               filter_max_iter=prm["filter_max_iter"])
    rel = np.abs(np.array(res.compliance) - g["compliance"]) / g["compliance"]
    assert rel[0] <= 1e-6 and rel.max() <= 1e-4
    assert np.abs(res.rho - g["rho"]).max() <= 1e-3


@pytest.mark.gpu
def test_gpu_learned_mixed_loop_with_finetuning(ctx, hx):
    """Mixed-precision learned FCG solves inside the device loop, with the
    networks fine-tuned every 5 iterations and the adaptive choice between
    learned and Jacobi solves: same compliance history as the oracle's FP64
    loop to the solver tolerance."""
    from importlib import import_module
    topopt = import_module(hx.__name__ + ".topopt")
    learned = import_module(hx.__name__ + ".learned")
    g, prm = _golden()
    dims = tuple(int(v) for v in g["dims"])
    nodes, el, bc, f = hx.workloads.cantilever(*dims)
    ctx.set_grid(*dims)
    learned.load_into(ctx)
    used = []
    res = topopt.run_oc_device(ctx, bc, f, prm["volfrac"], prm["radius"], 15, p=prm["p"],
                               e0=prm["e0"], emin=prm["emin"], nu=prm["nu"], move=prm["move"],
                               tol=prm["tol"], ref_compat=prm["ref_compat"],
                               filter_tol=prm["filter_tol"],
                               filter_max_iter=prm["filter_max_iter"], precision=1,
                               preconditioner=1, finetune_every=5,
                               callback=lambda it, c, rep: used.append(rep.fallback_used))
    rel = np.abs(np.array(res.compliance) - g["compliance"][:15]) / g["compliance"][:15]
    print(f"learned+mixed C0 loop: max rel compliance diff {rel.max():.2e}, "
          f"{len(res.finetune_ms)} fine-tunings, solve its {res.iterations}, "
          f"learned solves {res.pc_used}")
    assert rel.max() <= 1e-4
    assert len(res.finetune_ms) == 2 and res.pc_used[0] == 0 and res.pc_used[1] == 1
