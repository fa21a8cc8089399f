"""The reference's density update on the GPU (hx_update_density, the drop-in
for TopologyOptimization.update_density!, src/Optimization/TopOpt.jl:139-405)
against the oracle's float32 restatement (oracle.update_density).

Every per-element step runs in the reference's Float32 arithmetic on both
sides, so given the same filtered field the updated densities, the largest
change, the radius and the threshold are compared bit for bit (the device
reports its filtered field through filtered_out).  The filters themselves
(FP64 CG on both sides, summed in different orders) agree to 1e-9 before the
Float32 rounding, so the filtered fields are compared to 2 ulp.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIMS = (24, 10, 8)


def _config(dims=DIMS, h=(1.0, 1.0, 1.0), **opt):
    o = {"filter_R_init_perc": 8.0, "filter_R_interm_perc": 5.0, "filter_R_final_perc": 3.0}
    o.update(opt)
    return {"geometry": {"nElem_x_computed": dims[0], "nElem_y_computed": dims[1],
                         "nElem_z_computed": dims[2], "dx_computed": h[0], "dy_computed": h[1],
                         "dz_computed": h[2], "max_domain_dim": float(max(dims) * max(h))},
            "optimization_parameters": o, "solver_parameters": {"filter_tolerance": 1e-5}}


def _inputs(seed, n, protect=0.05):
    rng = np.random.default_rng(seed)
    dens = rng.uniform(0.05, 1.0, n).astype(np.float32)
    l1 = rng.gamma(2.0, 0.4, n).astype(np.float32)
    prot = rng.uniform(size=n) < protect
    orig = rng.uniform(0.5, 1.0, n).astype(np.float32)
    return dens, l1, prot, orig


def _run(hx, ctx, cfg, dens, l1, prot, orig, it, n_iter, E=1.0, allow=1.0, min_d=1e-3,
         max_d=1.0, dc=None):
    from importlib import import_module
    api = import_module(hx.__name__ + ".api")
    d = dens.copy()
    s = l1.copy()
    filt = np.empty_like(d)
    out = api.update_density(d, s, prot, E, allow, it, n_iter, orig, min_d, max_d, cfg, None,
                             False, dc=dc, filtered_out=filt, ctx=ctx)
    return d, s, filt, out


def _oracle(orc, cfg, dens, l1, prot, orig, it, n_iter, filtered=None, E=1.0, allow=1.0,
            min_d=1e-3, max_d=1.0):
    g = cfg["geometry"]
    o = cfg["optimization_parameters"]
    return orc.update_density(
        dens, l1, prot, E, allow, it, n_iter, orig, min_d, max_d,
        (g["nElem_x_computed"], g["nElem_y_computed"], g["nElem_z_computed"]),
        (g["dx_computed"], g["dy_computed"], g["dz_computed"]), g["max_domain_dim"],
        filter_tol=cfg["solver_parameters"]["filter_tolerance"],
        stress_regularization_ratio=o.get("stress_regularization_ratio", 0.0),
        R_init_perc=o.get("filter_R_init_perc", 0.0),
        R_interm_perc=o.get("filter_R_interm_perc", 0.0),
        R_final_perc=o.get("filter_R_final_perc", 0.0),
        R_interm_iter_perc=o.get("filter_R_interm_iter_perc", 50.0),
        final_density_threshold=o.get("final_density_threshold", 0.95),
        max_culling_ratio=o.get("max_culling_ratio", 0.1), filtered=filtered)


def _ulp_close(a, b, ulps=2):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    tol = ulps * np.spacing(np.maximum(np.abs(a), np.abs(b)))
    return bool(np.all(np.abs(a.astype(np.float64) - b) <= tol))


@pytest.mark.parametrize("it,n_iter", [(1, 40), (7, 40), (25, 40), (45, 40)])
def test_stress_ratio_update_matches_oracle(ctx, hx, orc, it, n_iter):
    n = int(np.prod(DIMS))
    dens, l1, prot, orig = _inputs(it, n)
    cfg = _config()
    d, s, filt, out = _run(hx, ctx, cfg, dens, l1, prot, orig, it, n_iter)
    # the filter against the oracle's (FP64 on both sides, then Float32)
    _, _, _, fo = _oracle(orc, cfg, dens, l1, prot, orig, it, n_iter)
    assert _ulp_close(filt, fo)
    # everything after the filter, bit for bit, on the device's filtered field
    do, so, (mc, R, thr, _, _), _ = _oracle(orc, cfg, dens, l1, prot, orig, it, n_iter,
                                            filtered=filt)
    assert np.array_equal(d, do)
    assert np.array_equal(s, l1)  # no stress regularisation: untouched
    assert out[0] == mc and out[1] == R and out[2] == thr
    assert out[4] > 0 and out[4] % 10 == 0 and out[5] < 1e-5
    assert np.array_equal(d[prot], orig[prot])


def test_culling_cap_ties_in_element_order(ctx, hx, orc):
    """A uniform stress field makes the filtered proposal nearly constant, so
    many candidates share a density value.  A first run gives the filtered
    field; the cap of the second run (same inputs, same field) is chosen so
    that the cut falls inside the longest run of equal candidate values.
    The reference's stable sort culls such ties in element order, and so
    must the device's radix select: the result equals the oracle's bit for
    bit and splits the run."""
    n = int(np.prod(DIMS))
    dens = np.full(n, 0.6, np.float32)
    l1 = np.full(n, 0.2, np.float32)
    prot = np.zeros(n, bool)
    prot[::97] = True
    orig = np.full(n, 0.8, np.float32)
    f32 = np.float32
    _, _, filt, _ = _run(hx, ctx, _config(), dens, l1, prot, orig, 40, 40)
    new = np.clip(filt, f32(1e-3), f32(1.0))
    cand = np.nonzero(~prot & (new > f32(1e-3)) & (new < f32(0.95)))[0]
    order = cand[np.argsort(new[cand], kind="stable")]
    vals = new[order]
    # the longest run of equal values among the sorted candidates
    starts = np.r_[0, np.nonzero(vals[1:] != vals[:-1])[0] + 1]
    ends = np.r_[starts[1:], vals.size]
    a, b = max(zip(starts, ends), key=lambda t: t[1] - t[0])
    assert b - a >= 3, "no run of tied candidates to split"
    active = np.count_nonzero(~prot & (new > f32(1e-3))) + np.count_nonzero(prot)
    k = a + (b - a) // 2  # cull the first k: the cut splits the run
    ratio = f32((k + 0.5) / active)
    assert int(np.floor(f32(active) * ratio)) == k
    cfg = _config(max_culling_ratio=float(ratio))
    d, _, filt2, out = _run(hx, ctx, cfg, dens, l1, prot, orig, 40, 40)
    assert np.array_equal(filt2, filt)  # deterministic
    do, _, (mc, R, thr, _, _), _ = _oracle(orc, cfg, dens, l1, prot, orig, 40, 40, filtered=filt)
    assert np.array_equal(d, do)
    culled = (d == f32(1e-3)) & ~prot
    assert np.count_nonzero(culled) == k
    run = order[a:b]
    assert 0 < np.count_nonzero(culled[run]) < run.size  # the run is split
    # ties go in element order: the culled members of the run come first
    assert np.all(culled[run][:k - a]) and not np.any(culled[run][k - a:])


def test_stress_regularisation_filters_the_l1_field_in_place(ctx, hx, orc):
    n = int(np.prod(DIMS))
    dens, l1, prot, orig = _inputs(3, n)
    cfg = _config(stress_regularization_ratio=1.5)
    d, s, filt, out = _run(hx, ctx, cfg, dens, l1, prot, orig, 10, 40)
    _, so, _, _ = _oracle(orc, cfg, dens, l1, prot, orig, 10, 40)
    assert not np.array_equal(s, l1) and _ulp_close(s, so)
    # the rest of the update from the device's filtered field
    cfg0 = _config(stress_regularization_ratio=0.0)
    do, _, (mc, R, thr, _, _), _ = _oracle(orc, cfg0, dens, s, prot, orig, 10, 40, filtered=filt)
    assert np.array_equal(d, do) and out[0] == mc and out[1] == R and out[2] == thr


def test_oc_mode_matches_oracle(ctx, hx, orc):
    n = int(np.prod(DIMS))
    dens, _, prot, orig = _inputs(5, n)
    rng = np.random.default_rng(6)
    dc = (-rng.uniform(0.1, 2.0, n)).astype(np.float32)
    cfg = _config(update="oc", volume_fraction=0.4, move_limit=0.2)
    d, s, filt, out = _run(hx, ctx, cfg, dens, np.zeros(n, np.float32), prot, orig, 3, 40, dc=dc)
    g = cfg["geometry"]
    conn0 = orc.structured_conn0(*DIMS)
    R, Reff = orc.radius_schedule(3, 40, (1.0, 1.0, 1.0), g["max_domain_dim"], 8.0, 5.0, 3.0)
    fo, _, _ = orc.helmholtz_filter(conn0, (DIMS[0] + 1) * (DIMS[1] + 1) * (DIMS[2] + 1),
                                    dc.astype(np.float64), 1.0, 1.0, 1.0,
                                    float(np.float32(Reff)), 1, float(np.float32(1e-5)), 200)
    assert _ulp_close(filt, fo.astype(np.float32))
    # the OC bisection runs on the FP64 filtered sensitivities on both sides
    xo, _, _ = orc.oc_update(dens.astype(np.float64), fo, np.ones(n), 0.4, 0.2)
    want = np.clip(xo.astype(np.float32), np.float32(1e-3), np.float32(1.0))
    want[prot] = orig[prot]
    assert _ulp_close(d, want, ulps=1)
    assert out[1] == R and out[2] == 0.0


def test_webdata_file_matches_the_restatement(ctx, hx, orc, tmp_path):
    """export_binary_for_web (src/IO/Postprocessing.jl:159-262) through
    hx_export_webdata: the file parses as load_checkpoint reads it and every
    array equals the oracle's float32 restatement bit for bit."""
    from importlib import import_module
    api = import_module(hx.__name__ + ".api")
    dims = (13, 7, 5)
    h = (1.0, 0.5, 2.0)
    nodes, el, _ = hx.mesh.generate_mesh(*dims, *h)
    n = el.shape[0]
    rng = np.random.default_rng(9)
    dens = rng.uniform(0.0, 1.0, n).astype(np.float32)
    l1 = rng.gamma(2.0, 1.0, n).astype(np.float32)
    pr = rng.standard_normal((3, n)).astype(np.float32)
    pr[:, ::11] = 0.0  # sign(0) = 0
    cfg = {"geometry": {"hole": {"type": "sphere", "stiffness_ratio": 0.0}},
           "optimization_parameters": {"max_culling_ratio": 0.1}, "external_forces": [1]}
    path = tmp_path / "it7.bin"
    cnt = api.export_binary_for_web(path, nodes, el, dens, l1, pr, None, np.float32(0.3), 7,
                                    np.float32(2.5), cfg, ctx=ctx)
    w = api.read_webdata(path)
    cent, d, s = orc.webdata_arrays(dims, h, dens, l1, pr.T, np.float32(0.3))
    assert cnt == w["count"] == d.size > 0
    assert w["magic"] == 0x48455841 and w["version"] == 2 and w["iter"] == 7
    assert w["radius"] == 2.5 and w["threshold"] == float(np.float32(0.3))
    assert w["h"] == h
    assert np.array_equal(w["centroids"], cent)
    assert np.array_equal(w["density"], d) and np.array_equal(w["signed_l1"], s)
    assert w["config"]["iteration"] == 7 and w["config"]["loads"] == [1]
    assert w["config"]["geometry"]["hole"]["action"] == "remove"
    c2, d2, it2, r2, t2 = api.load_checkpoint(path)
    assert it2 == 7 and np.array_equal(d2, d)
    # nothing passes the threshold: no file, as in the reference
    assert api.export_binary_for_web(tmp_path / "none.bin", nodes, el, dens * 0, l1, pr, None,
                                     np.float32(0.3), 7, np.float32(2.5), cfg, ctx=ctx) == 0
    assert not (tmp_path / "none.bin").exists()
