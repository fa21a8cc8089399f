"""Reference-shaped entry points: the names, arguments, return values and
error behaviour of the reference routines this library replaces.

  solve_system_gpu       src/Solvers/GPUSolver.jl:611-627
  apply_gpu_filter       src/Optimization/GPUHelmholtz.jl:344-376
  compute_stress_field   src/Core/Stress.jl:57-100
  update_density         src/Optimization/TopOpt.jl:139-405
  export_binary_for_web  src/IO/Postprocessing.jl:159-262 (and load_checkpoint,
                         src/IO/Configuration.jl:31-77, to read the file back)

Arrays follow the Julia layout (see mesh.py); each call runs on the GPU
through libhexat_b200.so.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import Context, HX_OK, HX_NOT_CONVERGED, HX_STALLED

_default_ctx = None


def default_context():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


# config["solver_parameters"]["preconditioner"] -> (preconditioner, precision,
# multigrid fallback) of the drop-in solve, as the reference reads it on every
# solve (src/Solvers/GPUSolver.jl:320-324; the multigrid preconditioner takes
# AMG's place)
_PRECONDITIONERS = {"jacobi": (_lib.HX_PC_JACOBI, _lib.HX_PREC_FP64, 0),
                    "jacobi_amg": (_lib.HX_PC_JACOBI, _lib.HX_PREC_FP64, 1),
                    "amg": (_lib.HX_PC_MULTIGRID, _lib.HX_PREC_FP64, 0)}


def _apply_solver_config(ctx, config):
    """Select the drop-in solver from the reference's config, if it names
    one (its default, as the reference's code default, is "jacobi")."""
    if not config:
        return
    sp = config.get("solver_parameters", {}) or {}
    if "preconditioner" not in sp:
        return
    name = str(sp["preconditioner"]).lower()
    if name not in _PRECONDITIONERS:
        raise ValueError(f"unknown preconditioner {sp['preconditioner']!r}")
    ctx.set_dropin_solver(*_PRECONDITIONERS[name])


def solve_system_gpu(nodes, elements, E, nu, bc_indicator, f, density, *, max_iter=40000,
                     tol=1e-6, method="native", solver="cg", use_precond=True,
                     shift_factor=1.0e-6, min_stiffness_threshold=1.0e-3, u_guess=None,
                     config=None, ctx=None):
    """GPUSolver.solve_system_gpu -> (x_full::float32[3nN], final_rel_res, prec_name).

    As in the reference, a solve whose every attempt fails still returns the
    best iterate (with a warning); bad input raises.  A config naming
    solver_parameters.preconditioner ("jacobi", "jacobi_amg", "amg") selects
    the solver as the reference does ("amg": the multigrid preconditioner)."""
    ctx = ctx or default_context()
    _apply_solver_config(ctx, config)
    nodes_cm = np.asfortranarray(nodes, dtype=np.float32)
    el_cm = np.asfortranarray(elements, dtype=np.int64)
    bc_cm = np.asfortranarray(bc_indicator, dtype=np.float32)
    f32 = np.ascontiguousarray(f, dtype=np.float32)
    d32 = np.ascontiguousarray(density, dtype=np.float32)
    nN, nE = nodes_cm.shape[0], el_cm.shape[0]
    ug = None
    if u_guess is not None and len(u_guess) == 3 * nN:
        ug = np.ascontiguousarray(u_guess, dtype=np.float32)
    x = np.zeros(3 * nN, np.float32)
    rel = C.c_double()
    name = C.create_string_buffer(32)
    st = ctx.lib.hx_solve_system_gpu(ctx.h, _p(nodes_cm), nN, _p(el_cm), nE, float(E), float(nu),
                                     _p(bc_cm), _p(f32), _p(d32), int(max_iter), float(tol),
                                     float(shift_factor), float(min_stiffness_threshold), _p(ug),
                                     _p(x), C.byref(rel), name, 32)
    if st not in (HX_OK, HX_STALLED, HX_NOT_CONVERGED, _lib.HX_BREAKDOWN, _lib.HX_DIVERGED,
                  _lib.HX_NONFINITE):
        ctx.check(st, "solve_system_gpu")
    if st not in (HX_OK, HX_STALLED):
        import warnings
        warnings.warn("All solver attempts failed. Returning best stagnated result.")
    return x, rel.value, name.value.decode()


def solve_system_grid(nelem, h, E, nu, bc_indicator, f, density, *, max_iter=40000, tol=1e-6,
                      shift_factor=1.0e-6, min_stiffness_threshold=1.0e-3, u_guess=None,
                      ctx=None):
    """solve_system_gpu on the unpruned generate_mesh grid (nelem = (nx, ny,
    nz), h = (dx, dy, dz)) with the pruning of src/Solvers/Solver.jl:60-91
    done on the device -> (x_full::float32[3nN], final_rel_res, prec_name).
    The result equals the reference's prune / solve / reconstruct path."""
    ctx = ctx or default_context()
    bc_cm = np.asfortranarray(bc_indicator, dtype=np.float32)
    f32 = np.ascontiguousarray(f, dtype=np.float32)
    d32 = np.ascontiguousarray(density, dtype=np.float32)
    ug = None if u_guess is None else np.ascontiguousarray(u_guess, dtype=np.float32)
    x = np.zeros(f32.shape[0], np.float32)
    rel = C.c_double()
    name = C.create_string_buffer(32)
    st = ctx.lib.hx_solve_system_grid(ctx.h, int(nelem[0]), int(nelem[1]), int(nelem[2]),
                                      float(h[0]), float(h[1]), float(h[2]), float(E), float(nu),
                                      _p(bc_cm), _p(f32), _p(d32), int(max_iter), float(tol),
                                      float(shift_factor), float(min_stiffness_threshold),
                                      _p(ug), _p(x), C.byref(rel), name, 32)
    if st not in (HX_OK, HX_STALLED, HX_NOT_CONVERGED, _lib.HX_BREAKDOWN, _lib.HX_DIVERGED,
                  _lib.HX_NONFINITE):
        ctx.check(st, "solve_system_grid")
    if st not in (HX_OK, HX_STALLED):
        import warnings
        warnings.warn("All solver attempts failed. Returning best stagnated result.")
    return x, rel.value, name.value.decode()


def apply_gpu_filter(density, nelem_x, nelem_y, nelem_z, dx, dy, dz, radius, elements=None,
                     tol=1.0e-5, ref_compat=1, ctx=None):
    """GPUHelmholtz.apply_gpu_filter! -> (filtered, time_s, iters, res).

    `elements` is accepted for signature parity; the filter always runs on the
    full structured grid, as the reference's does.  ref_compat=1 (default)
    reproduces the reference element (1.5*dz tall).  On failure the result is
    an empty float32 array, which the reference's caller reads as "failed"."""
    ctx = ctx or default_context()
    d32 = np.ascontiguousarray(density, dtype=np.float32)
    out = np.empty_like(d32)
    t = C.c_double()
    it = C.c_int32()
    res = C.c_double()
    st = ctx.lib.hx_apply_gpu_filter(ctx.h, _p(d32), int(nelem_x), int(nelem_y), int(nelem_z),
                                     float(dx), float(dy), float(dz), float(radius), float(tol),
                                     int(ref_compat), _p(out), C.byref(t), C.byref(it),
                                     C.byref(res))
    if st != HX_OK:
        return np.empty(0, np.float32), 0.0, 0, 0.0
    return out, t.value, it.value, res.value


def compute_stress_field(nodes, elements, U, E, nu, density, ctx=None):
    """Stress.compute_stress_field -> (principal (3,nE), vonmises (nE,),
    voigt (6,nE), l1 (nE,), principal_dir (3,nE)), float32, Julia-shaped."""
    ctx = ctx or default_context()
    nodes_cm = np.asfortranarray(nodes, dtype=np.float32)
    el_cm = np.asfortranarray(elements, dtype=np.int64)
    nN, nE = nodes_cm.shape[0], el_cm.shape[0]
    u32 = np.ascontiguousarray(U, dtype=np.float32)
    d32 = np.ascontiguousarray(density, dtype=np.float32)
    pr = np.empty((nE, 3), np.float32)
    vm = np.empty(nE, np.float32)
    vo = np.empty((nE, 6), np.float32)
    l1 = np.empty(nE, np.float32)
    dr = np.empty((nE, 3), np.float32)
    st = ctx.lib.hx_compute_stress_field(ctx.h, _p(nodes_cm), nN, _p(el_cm), nE, _p(u32),
                                         float(E), float(nu), _p(d32), _p(pr), _p(vm), _p(vo),
                                         _p(l1), _p(dr))
    ctx.check(st, "compute_stress_field")
    return pr.T, vm, vo.T, l1, dr.T


def update_params(config, mode=None):
    """hx_update_params from the reference's config Dict (the keys
    update_density! reads, src/Optimization/TopOpt.jl:156-169,216-222,351-352,
    with its defaults); mode "stress_ratio" (the reference, default) or "oc"
    (config["optimization_parameters"]["update"], or the argument)."""
    o = config.get("optimization_parameters", {})
    g = config["geometry"]
    sp = config.get("solver_parameters", {})
    p = _lib.UpdateParams()
    _lib.load().hx_default_update_params(C.byref(p))
    p.nelem[:] = [int(g["nElem_x_computed"]), int(g["nElem_y_computed"]),
                  int(g["nElem_z_computed"])]
    p.h[:] = [float(g["dx_computed"]), float(g["dy_computed"]), float(g["dz_computed"])]
    p.max_domain_dim = float(g["max_domain_dim"])
    p.filter_tolerance = float(sp.get("filter_tolerance", 1.0e-5))
    p.stress_regularization_ratio = float(o.get("stress_regularization_ratio", 0.0))
    p.filter_R_init_perc = float(o.get("filter_R_init_perc", 0.0))
    p.filter_R_interm_perc = float(o.get("filter_R_interm_perc", 0.0))
    p.filter_R_final_perc = float(o.get("filter_R_final_perc", 0.0))
    p.filter_R_interm_iter_perc = float(o.get("filter_R_interm_iter_perc", 50.0))
    p.final_density_threshold = float(o.get("final_density_threshold", 0.95))
    p.max_culling_ratio = float(o.get("max_culling_ratio", 0.1))
    mode = mode or o.get("update", "stress_ratio")
    if mode not in ("stress_ratio", "oc"):
        raise ValueError(f"unknown update mode {mode!r}")
    p.mode = _lib.HX_UPDATE_OC if mode == "oc" else _lib.HX_UPDATE_STRESS_RATIO
    p.oc_volfrac = float(o.get("volume_fraction", 0.3))
    p.oc_move = float(o.get("move_limit", 0.2))
    return p


def update_density(density, l1_stress_norm_field, protected_elements_mask, E,
                   l1_stress_allowable, iter, number_of_iterations, original_density,
                   min_density, max_density, config, elements=None, is_annealing=False, *,
                   dc=None, filtered_out=None, ctx=None):
    """TopologyOptimization.update_density! -> (max_change, R_length,
    current_threshold, filter_time, filter_iters, filter_res).

    `density` (and `l1_stress_norm_field`, when stress regularisation is on)
    are float32 arrays updated in place, as the Julia vectors are; `elements`
    and `is_annealing` are accepted for signature parity (the update runs on
    the structured grid the config names, as the reference's filter does).
    With config["optimization_parameters"]["update"] == "oc" the OC step
    runs instead, on the sensitivities `dc`."""
    ctx = ctx or default_context()
    for name, a in (("density", density), ("l1_stress_norm_field", l1_stress_norm_field)):
        if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
            raise TypeError(f"{name} must be a contiguous float32 array (updated in place)")
    prot = np.ascontiguousarray(np.asarray(protected_elements_mask, dtype=bool), dtype=np.uint8)
    orig = np.ascontiguousarray(original_density, dtype=np.float32)
    dcv = None if dc is None else np.ascontiguousarray(dc, dtype=np.float32)
    p = update_params(config)
    res = _lib.UpdateResult()
    st = ctx.lib.hx_update_density(ctx.h, _p(density), _p(l1_stress_norm_field), _p(prot),
                                   float(E), float(l1_stress_allowable), int(iter),
                                   int(number_of_iterations), _p(orig), float(min_density),
                                   float(max_density), C.byref(p), _p(dcv), _p(filtered_out),
                                   C.byref(res))
    ctx.check(st, "update_density")
    return (res.max_change, res.R_length, res.current_threshold, res.filter_time,
            res.filter_iters, res.filter_res)


def _webdata_meta(config, iter, current_radius, threshold):
    """The JSON metadata export_binary_for_web writes (Postprocessing.jl:198-231):
    the config plus iteration, radius and threshold, an 'action' synthesised
    from 'stiffness_ratio' for geometry shapes, and the loads / bcs / settings
    aliases the viewers read."""
    import copy
    meta = copy.deepcopy(config)
    meta["iteration"] = int(iter)
    meta["radius"] = float(current_radius)
    meta["threshold"] = float(threshold)
    geom = meta.get("geometry")
    if isinstance(geom, dict):
        for shape in geom.values():
            if isinstance(shape, dict) and "type" in shape and "action" not in shape \
                    and "stiffness_ratio" in shape:
                shape["action"] = "add" if float(shape["stiffness_ratio"]) > 0 else "remove"
    meta["loads"] = config.get("external_forces", [])
    meta["bcs"] = config.get("boundary_conditions", [])
    meta["settings"] = config.get("optimization_parameters", {})
    return meta


def export_binary_for_web(filename, nodes, elements, density, l1_stress, principal_field, geom,
                          threshold, iter, current_radius, config, ctx=None):
    """export_binary_for_web: writes the webdata/checkpoint file.  `nodes`
    and `elements` must be generate_mesh's (grid numbering); `geom` is
    accepted for signature parity (the element sizes come from the mesh);
    principal_field is (3, nE) as in the reference.  Returns the number of
    elements written (0: no file, as in the reference)."""
    import json
    ctx = ctx or default_context()
    ctx.set_mesh(nodes, elements)
    d = np.ascontiguousarray(density, dtype=np.float32)
    l1 = np.ascontiguousarray(l1_stress, dtype=np.float32)
    pr = np.ascontiguousarray(np.asarray(principal_field, dtype=np.float32).T)
    text = json.dumps(_webdata_meta(config, iter, current_radius, threshold),
                      separators=(",", ":")).encode()
    cnt = C.c_int64()
    st = ctx.lib.hx_export_webdata(ctx.h, str(filename).encode(), _lib.HX_F32, _p(d), _p(l1),
                                   _p(pr), float(threshold), int(iter), float(current_radius),
                                   text, len(text), C.byref(cnt))
    ctx.check(st, "export_binary_for_web")
    return cnt.value


def read_webdata(filename):
    """Every field of a webdata file, in the layout load_checkpoint
    (src/IO/Configuration.jl:31-77) reads: a dict with magic, version, iter,
    radius, threshold, count, h, centroids (count, 3), density, signed_l1 and
    config (the parsed JSON)."""
    import json
    with open(filename, "rb") as fh:
        buf = fh.read()
    hdr = np.frombuffer(buf, "<u4", 2, 0)
    it = int(np.frombuffer(buf, "<i4", 1, 8)[0])
    rad, thr = (float(v) for v in np.frombuffer(buf, "<f4", 2, 12))
    count = int(np.frombuffer(buf, "<u4", 1, 20)[0])
    h = tuple(float(v) for v in np.frombuffer(buf, "<f4", 3, 24))
    o = 36
    cent = np.frombuffer(buf, "<f4", 3 * count, o).reshape(count, 3)
    o += 12 * count
    dens = np.frombuffer(buf, "<f4", count, o)
    o += 4 * count
    sl1 = np.frombuffer(buf, "<f4", count, o)
    o += 4 * count
    jl = int(np.frombuffer(buf, "<u4", 1, o)[0])
    o += 4
    cfg = json.loads(buf[o:o + jl].decode()) if jl else None
    assert o + jl == len(buf), "trailing bytes in webdata file"
    return {"magic": int(hdr[0]), "version": int(hdr[1]), "iter": it, "radius": rad,
            "threshold": thr, "count": count, "h": h, "centroids": cent, "density": dens,
            "signed_l1": sl1, "config": cfg}


def load_checkpoint(filename):
    """load_checkpoint (src/IO/Configuration.jl:31-77) -> (config, density,
    restart_iter, restart_radius, restart_threshold)."""
    w = read_webdata(filename)
    if w["magic"] != 0x48455841:
        raise ValueError("Invalid file format. Not a HEXA checkpoint.")
    return w["config"], w["density"].copy(), w["iter"], w["radius"], w["threshold"]
