"""Reference-shaped entry points: the names, arguments, return values and
error behaviour of the reference routines this library replaces.

  solve_system_gpu       src/Solvers/GPUSolver.jl:611-627
  apply_gpu_filter       src/Optimization/GPUHelmholtz.jl:344-376
  compute_stress_field   src/Core/Stress.jl:57-100

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


def solve_system_gpu(nodes, elements, E, nu, bc_indicator, f, density, *, max_iter=40000,
                     tol=1e-6, method="native", solver="cg", use_precond=True,
                     shift_factor=1.0e-6, min_stiffness_threshold=1.0e-3, u_guess=None,
                     config=None, ctx=None):
    """GPUSolver.solve_system_gpu -> (x_full::float32[3nN], final_rel_res, prec_name).

    As in the reference, a solve whose every attempt fails still returns the
    best iterate (with a warning); bad input raises."""
    ctx = ctx or default_context()
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
