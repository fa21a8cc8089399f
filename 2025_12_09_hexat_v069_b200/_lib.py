"""ctypes binding of libhexat_b200.so (the C ABI declared in include/hexat_b200.h).

The shared library is the product: every numerical call goes to the GPU
through it.  Loading fails loudly when the library has not been built; there
is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhexat_b200.so")

HX_OK, HX_NOT_CONVERGED, HX_STALLED, HX_BREAKDOWN, HX_NONFINITE = 0, 1, 2, 3, 4
HX_OOM, HX_BAD_ARG, HX_CUDA_ERROR, HX_NO_DEVICE, HX_DIVERGED = 5, 6, 7, 8, 9
HX_F32, HX_F64 = 0, 1
HX_PREC_FP64, HX_PREC_MIXED32 = 0, 1
HX_PC_JACOBI, HX_PC_LEARNED, HX_PC_NONE, HX_PC_MULTIGRID = 0, 1, 2, 3
(HX_KERNEL_PCG_STEP_FP64, HX_KERNEL_PCG_UPDATE_FP64, HX_KERNEL_APPLY_FP64, HX_KERNEL_PCG_STEP_FP32,
 HX_KERNEL_FILTER_MATVEC, HX_KERNEL_CONV3, HX_KERNEL_NET_APPLY, HX_KERNEL_FCG_STEP_FP32) = range(8)


class SolveOpts(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("preconditioner", C.c_int32), ("tol", C.c_double),
        ("max_iter", C.c_int32), ("warm_start", C.c_int32), ("shift_factor", C.c_double),
        ("wall_limit_ms", C.c_double), ("check_every", C.c_int32), ("keep_best", C.c_int32),
        ("inner_tol", C.c_double), ("max_refine", C.c_int32), ("ref_retry", C.c_int32),
        ("divergence_checks", C.c_int32), ("verify_true_residual", C.c_int32),
        ("learned_no_fallback", C.c_int32), ("multigrid_fallback", C.c_int32),
        ("mg_smooth_degree", C.c_int32), ("reserved", C.c_int32 * 3),
    ]


class SolveReport(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iterations", C.c_int32), ("refinements", C.c_int32),
        ("attempts", C.c_int32), ("fallback_used", C.c_int32), ("zero_rhs", C.c_int32),
        ("rel_res", C.c_double), ("true_rel_res", C.c_double), ("shift", C.c_double),
        ("time_setup_ms", C.c_double), ("time_solve_ms", C.c_double),
        ("time_total_ms", C.c_double), ("time_device_ms", C.c_double),
        ("kernel_launches", C.c_double), ("time_precond_setup_ms", C.c_double),
        ("reserved", C.c_double * 1),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class UpdateParams(C.Structure):
    _fields_ = [
        ("nelem", C.c_int64 * 3), ("h", C.c_double * 3), ("max_domain_dim", C.c_double),
        ("filter_tolerance", C.c_double), ("stress_regularization_ratio", C.c_double),
        ("filter_R_init_perc", C.c_double), ("filter_R_interm_perc", C.c_double),
        ("filter_R_final_perc", C.c_double), ("filter_R_interm_iter_perc", C.c_double),
        ("final_density_threshold", C.c_double), ("max_culling_ratio", C.c_double),
        ("mode", C.c_int32), ("reserved0", C.c_int32), ("oc_volfrac", C.c_double),
        ("oc_move", C.c_double), ("reserved", C.c_double * 4),
    ]


class UpdateResult(C.Structure):
    _fields_ = [
        ("max_change", C.c_double), ("R_length", C.c_double), ("current_threshold", C.c_double),
        ("filter_time", C.c_double), ("filter_res", C.c_double), ("filter_iters", C.c_int32),
        ("culled", C.c_int32), ("reserved", C.c_double * 2),
    ]


HX_UPDATE_STRESS_RATIO, HX_UPDATE_OC = 0, 1

_vp, _i32, _i64, _dbl, _f32p, _i64p = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_void_p, C.c_void_p

# name -> (restype, argtypes); the full exported surface of include/hexat_b200.h
PROTOTYPES = {
    "hx_create": (_i32, [C.POINTER(_vp), _i32]),
    "hx_destroy": (None, [_vp]),
    "hx_last_error": (C.c_char_p, [_vp]),
    "hx_default_opts": (None, [C.POINTER(SolveOpts)]),
    "hx_status_string": (C.c_char_p, [_i32]),
    "hx_get_stream": (_i32, [_vp, C.POINTER(_vp)]),
    "hx_kernel_launches": (_i64, [_vp]),
    "hx_time_kernel": (_i32, [_vp, _i32, _i32, C.POINTER(_dbl)]),
    "hx_set_grid": (_i32, [_vp, _i64, _i64, _i64, _dbl, _dbl, _dbl]),
    "hx_set_mesh": (_i32, [_vp, _f32p, _i64, _i64p, _i64]),
    "hx_set_material": (_i32, [_vp, _dbl, _dbl]),
    "hx_set_bc": (_i32, [_vp, _f32p, _i64]),
    "hx_get_grid": (_i32, [_vp, _vp, _vp]),
    "hx_apply_stiffness": (_i32, [_vp, _i32, _vp, _vp, _vp]),
    "hx_diagonal": (_i32, [_vp, _i32, _vp, _vp]),
    "hx_apply_stiffness_noalloc": (_i32, [_i64, _i64, _i64, _dbl, _dbl, _dbl, _dbl, _vp, _vp, _vp,
                                          _vp, _vp]),
    "hx_solve": (_i32, [_vp, _i32, _vp, _vp, _vp, C.POINTER(SolveOpts), C.POINTER(SolveReport)]),
    "hx_solve_device": (_i32, [_vp, _vp, _vp, _vp, C.POINTER(SolveOpts), C.POINTER(SolveReport)]),
    "hx_solve_system_gpu": (_i32, [_vp, _f32p, _i64, _i64p, _i64, C.c_float, C.c_float, _f32p,
                                   _f32p, _f32p, _i32, _dbl, C.c_float, C.c_float, _f32p, _f32p,
                                   C.POINTER(_dbl), C.c_char_p, _i32]),
    "hx_solve_system_grid": (_i32, [_vp, _i64, _i64, _i64, _dbl, _dbl, _dbl, C.c_float,
                                    C.c_float, _f32p, _f32p, _f32p, _i32, _dbl, C.c_float,
                                    C.c_float, _f32p, _f32p, C.POINTER(_dbl), C.c_char_p, _i32]),
    "hx_export_webdata": (_i32, [_vp, C.c_char_p, _i32, _vp, _vp, _vp, C.c_float, _i32,
                                 C.c_float, C.c_char_p, _i64, C.POINTER(_i64)]),
    "hx_export_webdata_device": (_i32, [_vp, C.c_char_p, _vp, _vp, _vp, C.c_float, _i32,
                                        C.c_float, C.c_char_p, _i64, C.POINTER(_i64)]),
    "hx_filter": (_i32, [_vp, _i32, _vp, _vp, _dbl, _i32, _dbl, _i32, C.POINTER(SolveReport)]),
    "hx_filter_device": (_i32, [_vp, _vp, _vp, _dbl, _i32, _dbl, _i32, C.POINTER(SolveReport)]),
    "hx_apply_gpu_filter": (_i32, [_vp, _f32p, _i64, _i64, _i64, _dbl, _dbl, _dbl, _dbl, _dbl,
                                   _i32, _f32p, C.POINTER(_dbl), C.POINTER(_i32),
                                   C.POINTER(_dbl)]),
    "hx_stress": (_i32, [_vp, _i32, _vp, _vp, _dbl, _dbl, _vp, _vp, _vp, _vp, _vp]),
    "hx_compute_stress_field": (_i32, [_vp, _f32p, _i64, _i64p, _i64, _f32p, C.c_float,
                                       C.c_float, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]),
    "hx_compliance": (_i32, [_vp, _i32, _vp, _vp, C.POINTER(_dbl)]),
    "hx_net_init": (_i32, [_vp, C.c_uint64]),
    "hx_net_set_params": (_i32, [_vp, _vp]),
    "hx_net_get_params": (_i32, [_vp, _vp]),
    "hx_net_forward_backward": (_i32, [_vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp]),
    "hx_net_prepare": (_i32, [_vp, _vp]),
    "hx_net_apply": (_i32, [_vp, _vp, _vp]),
    "hx_gmg_apply": (_i32, [_vp, _vp, _vp]),
    "hx_set_dropin_solver": (_i32, [_vp, C.c_int32, C.c_int32, C.c_int32]),
    "hx_selftest_wait_timeout": (_i32, [_vp, C.POINTER(_i32)]),
    "hx_simp_device": (_i32, [_vp, _vp, _dbl, _dbl, _dbl, _vp]),
    "hx_sensitivity_device": (_i32, [_vp, _vp, _vp, _dbl, _dbl, _dbl, _vp]),
    "hx_compliance_device": (_i32, [_vp, _vp, _vp, C.POINTER(_dbl)]),
    "hx_oc_update_device": (_i32, [_vp, _vp, _vp, _vp, _dbl, _dbl, _vp, C.POINTER(_dbl),
                                   C.POINTER(_i32)]),
    "hx_stress_pnorm": (_i32, [_vp, _i32, _vp, _vp, _dbl, _dbl, _dbl, C.POINTER(_dbl),
                               C.POINTER(_dbl)]),
    "hx_net_train_step": (_i32, [_vp, _vp, _vp, _dbl, _i32, C.POINTER(_dbl)]),
    "hx_net_train_batch": (_i32, [_vp, _vp, _vp, _i32, _dbl, _i32, C.POINTER(_dbl)]),
    "hx_pcg_snapshots": (_i32, [_vp, _vp, _vp, _i32, _i32, _dbl, _vp, C.POINTER(_i32)]),
    "hx_residual_device": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "hx_element_energy": (_i32, [_vp, _i32, _vp, _vp]),
    "hx_oc_update": (_i32, [_vp, _i32, _vp, _vp, _vp, _dbl, _dbl, _vp, C.POINTER(_dbl),
                            C.POINTER(_i32)]),
    "hx_default_update_params": (None, [C.POINTER(UpdateParams)]),
    "hx_update_density": (_i32, [_vp, _vp, _vp, _vp, C.c_float, C.c_float, _i32, _i32, _vp,
                                 C.c_float, C.c_float, C.POINTER(UpdateParams), _vp, _vp,
                                 C.POINTER(UpdateResult)]),
}

_lib = None


def header_symbols():
    """Function names declared with HX_API in include/hexat_b200.h."""
    import re
    path = os.path.join(os.path.dirname(HERE), "include", "hexat_b200.h")
    with open(path) as fh:
        txt = fh.read()
    return sorted(set(re.findall(r"HX_API\s+[\w\s\*]+?\b(hx_\w+)\s*\(", txt)))


def load(path=LIB_PATH):
    """Load the library (once) and attach prototypes.  Raises if missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m ...build` (nvcc, sm_100a); "
            "there is no CPU fallback")
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class HexatError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} [status {status}]")
        self.status = status


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _dtype_code(a):
    if a.dtype == np.float64:
        return HX_F64
    if a.dtype == np.float32:
        return HX_F32
    raise TypeError("arrays must be float32 or float64")


def default_opts(**kw):
    o = SolveOpts()
    load().hx_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class Context:
    """One library context (CUDA stream + cached device buffers) on a device."""

    def __init__(self, device=0):
        self.lib = load()
        h = C.c_void_p()
        st = self.lib.hx_create(C.byref(h), int(device))
        if st != HX_OK:
            raise HexatError(st, f"hx_create failed: {self.lib.hx_status_string(st).decode()}")
        self.h = h
        self.dims = None

    def close(self):
        if self.h:
            self.lib.hx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def check(self, st, what, ok=(HX_OK,)):
        if st not in ok:
            msg = self.lib.hx_last_error(self.h).decode()
            raise HexatError(st, f"{what}: {self.lib.hx_status_string(st).decode()}: {msg}")
        return st

    # ---- mesh / material / BC ----
    def set_grid(self, nx, ny, nz, dx=1.0, dy=1.0, dz=1.0):
        self.check(self.lib.hx_set_grid(self.h, nx, ny, nz, dx, dy, dz), "hx_set_grid")
        self.dims = (nx, ny, nz)

    def set_mesh(self, nodes, elements):
        """nodes: (nN,3) float32; elements: (nE,8) int 1-based (Julia layout)."""
        nodes_cm = np.asfortranarray(nodes, dtype=np.float32)
        el_cm = np.asfortranarray(elements, dtype=np.int64)
        self.check(self.lib.hx_set_mesh(self.h, _ptr(nodes_cm), nodes_cm.shape[0], _ptr(el_cm),
                                        el_cm.shape[0]), "hx_set_mesh")
        self.dims = self.grid()[0]

    def grid(self):
        d = (C.c_int64 * 3)()
        h = (C.c_double * 3)()
        self.check(self.lib.hx_get_grid(self.h, d, h), "hx_get_grid")
        return tuple(d), tuple(h)

    def set_material(self, E, nu):
        self.check(self.lib.hx_set_material(self.h, E, nu), "hx_set_material")

    def set_bc(self, bc_indicator):
        bc = np.asfortranarray(bc_indicator, dtype=np.float32)
        self.check(self.lib.hx_set_bc(self.h, _ptr(bc), bc.shape[0]), "hx_set_bc")

    # ---- operator ----
    def apply_stiffness(self, x, factor):
        x = np.ascontiguousarray(x)
        factor = np.ascontiguousarray(factor, dtype=x.dtype)
        y = np.empty_like(x)
        self.check(self.lib.hx_apply_stiffness(self.h, _dtype_code(x), _ptr(x), _ptr(factor),
                                               _ptr(y)), "hx_apply_stiffness")
        return y

    def diagonal(self, factor, n_dofs):
        factor = np.ascontiguousarray(factor)
        d = np.empty(n_dofs, dtype=factor.dtype)
        self.check(self.lib.hx_diagonal(self.h, _dtype_code(factor), _ptr(factor), _ptr(d)),
                   "hx_diagonal")
        return d

    # ---- solve ----
    def solve(self, f, factor, u0=None, opts=None, ok=(HX_OK,), **kw):
        f = np.ascontiguousarray(f)
        factor = np.ascontiguousarray(factor, dtype=f.dtype)
        o = opts if opts is not None else default_opts(**kw)
        if u0 is not None:
            u = np.ascontiguousarray(u0, dtype=f.dtype).copy()
            o.warm_start = 1
        else:
            u = np.zeros_like(f)
        rep = SolveReport()
        st = self.lib.hx_solve(self.h, _dtype_code(f), _ptr(f), _ptr(factor), _ptr(u),
                               C.byref(o), C.byref(rep))
        self.check(st, "hx_solve", ok)
        return u, rep

    def solve_device(self, f_ptr, fac_ptr, u_ptr, opts=None, ok=(HX_OK,), **kw):
        o = opts if opts is not None else default_opts(**kw)
        rep = SolveReport()
        st = self.lib.hx_solve_device(self.h, C.c_void_p(f_ptr), C.c_void_p(fac_ptr),
                                      C.c_void_p(u_ptr), C.byref(o), C.byref(rep))
        self.check(st, "hx_solve_device", ok)
        return rep

    # ---- instrumentation ----
    def stream(self):
        s = C.c_void_p()
        self.check(self.lib.hx_get_stream(self.h, C.byref(s)), "hx_get_stream")
        return s.value

    def kernel_launches(self):
        return int(self.lib.hx_kernel_launches(self.h))

    def time_kernel(self, kernel, reps=20):
        ms = C.c_double()
        self.check(self.lib.hx_time_kernel(self.h, int(kernel), int(reps), C.byref(ms)),
                   "hx_time_kernel")
        return ms.value

    # ---- learned preconditioner ----
    NET_PARAMS = 3 * 4 * 27 * 256
    NET_FIRST_LEVEL = 2  # HX_NET_FIRST_LEVEL

    def net_init(self, seed=1):
        self.check(self.lib.hx_net_init(self.h, int(seed)), "hx_net_init")

    def net_set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == self.NET_PARAMS
        self.check(self.lib.hx_net_set_params(self.h, _ptr(p)), "hx_net_set_params")

    def net_get_params(self):
        p = np.empty(self.NET_PARAMS, np.float32)
        self.check(self.lib.hx_net_get_params(self.h, _ptr(p)), "hx_net_get_params")
        return p

    def net_forward_backward(self, dims, x0, dy):
        x0 = np.ascontiguousarray(x0, dtype=np.float32)
        dy = np.ascontiguousarray(dy, dtype=np.float32)
        y = np.empty_like(x0)
        g = np.empty(self.NET_PARAMS, np.float32)
        self.check(self.lib.hx_net_forward_backward(self.h, *dims, _ptr(x0), _ptr(dy), _ptr(y),
                                                    _ptr(g)), "hx_net_forward_backward")
        return y, g

    def net_prepare(self, fac_ptr):
        self.check(self.lib.hx_net_prepare(self.h, C.c_void_p(fac_ptr)), "hx_net_prepare")

    def selftest_wait_timeout(self):
        """True when a convolution CTA's bounded wait ran out and was reported
        (see hx_selftest_wait_timeout)."""
        d = C.c_int32()
        self.check(self.lib.hx_selftest_wait_timeout(self.h, C.byref(d)),
                   "hx_selftest_wait_timeout")
        return bool(d.value)

    def net_apply(self, r_ptr, z_ptr):
        self.check(self.lib.hx_net_apply(self.h, C.c_void_p(r_ptr), C.c_void_p(z_ptr)),
                   "hx_net_apply")

    def set_dropin_solver(self, preconditioner=HX_PC_JACOBI, precision=HX_PREC_FP64,
                          multigrid_fallback=1):
        """Solver of this context's drop-in solves (api.solve_system_gpu /
        solve_system_grid); the default is the reference's "jacobi_amg"."""
        self.check(self.lib.hx_set_dropin_solver(self.h, int(preconditioner), int(precision),
                                                 int(multigrid_fallback)),
                   "hx_set_dropin_solver")

    def gmg_apply(self, r_ptr, z_ptr):
        self.check(self.lib.hx_gmg_apply(self.h, C.c_void_p(r_ptr), C.c_void_p(z_ptr)),
                   "hx_gmg_apply")

    def net_train_step(self, r_ptr, e_ptr, lr, loss_kind=0):
        loss = C.c_double()
        self.check(self.lib.hx_net_train_step(self.h, C.c_void_p(r_ptr), C.c_void_p(e_ptr or 0),
                                              float(lr), int(loss_kind), C.byref(loss)),
                   "hx_net_train_step")
        return loss.value

    def net_train_batch(self, r_ptrs, e_ptrs, lr, loss_kind=0):
        """One Adam step on the summed gradient of the pairs (device pointers)."""
        k = len(r_ptrs)
        ra = (C.c_void_p * k)(*[C.c_void_p(p) for p in r_ptrs])
        ea = (C.c_void_p * k)(*[C.c_void_p(p) for p in e_ptrs]) if e_ptrs is not None else None
        loss = C.c_double()
        self.check(self.lib.hx_net_train_batch(self.h, ra, ea, k, float(lr), int(loss_kind),
                                               C.byref(loss)), "hx_net_train_batch")
        return loss.value

    def pcg_snapshots(self, f_ptr, fac_ptr, every, count, tol, snaps_ptr):
        taken = C.c_int32()
        self.check(self.lib.hx_pcg_snapshots(self.h, C.c_void_p(f_ptr), C.c_void_p(fac_ptr),
                                             int(every), int(count), float(tol),
                                             C.c_void_p(snaps_ptr), C.byref(taken)),
                   "hx_pcg_snapshots")
        return taken.value

    def residual_device(self, f_ptr, fac_ptr, x_ptr, r_ptr):
        self.check(self.lib.hx_residual_device(self.h, C.c_void_p(f_ptr), C.c_void_p(fac_ptr),
                                               C.c_void_p(x_ptr), C.c_void_p(r_ptr)),
                   "hx_residual_device")

    # ---- filter ----
    def filter(self, rho, radius, ref_compat=0, tol=1e-5, max_iter=200):
        rho = np.ascontiguousarray(rho)
        out = np.empty_like(rho)
        rep = SolveReport()
        self.check(self.lib.hx_filter(self.h, _dtype_code(rho), _ptr(rho), _ptr(out),
                                      float(radius), int(ref_compat), float(tol), int(max_iter),
                                      C.byref(rep)), "hx_filter")
        return out, rep

    def filter_device(self, rho_ptr, out_ptr, radius, ref_compat=0, tol=1e-5, max_iter=200):
        rep = SolveReport()
        self.check(self.lib.hx_filter_device(self.h, C.c_void_p(rho_ptr), C.c_void_p(out_ptr),
                                             float(radius), int(ref_compat), float(tol),
                                             int(max_iter), C.byref(rep)), "hx_filter_device")
        return rep

    # ---- stress / OC ----
    def stress(self, u, density, E, nu):
        u = np.ascontiguousarray(u)
        density = np.ascontiguousarray(density, dtype=u.dtype)
        ne = density.shape[0]
        pr = np.empty((ne, 3), u.dtype)
        vm = np.empty(ne, u.dtype)
        vo = np.empty((ne, 6), u.dtype)
        l1 = np.empty(ne, u.dtype)
        dr = np.empty((ne, 3), u.dtype)
        self.check(self.lib.hx_stress(self.h, _dtype_code(u), _ptr(u), _ptr(density), E, nu,
                                      _ptr(pr), _ptr(vm), _ptr(vo), _ptr(l1), _ptr(dr)),
                   "hx_stress")
        return pr, vm, vo, l1, dr

    # ---- device-resident loop pieces (device pointers, grid numbering) ----
    def simp_device(self, rho_ptr, fac_ptr, p=3.0, e0=1.0, emin=1e-9):
        self.check(self.lib.hx_simp_device(self.h, C.c_void_p(rho_ptr), p, e0, emin,
                                           C.c_void_p(fac_ptr)), "hx_simp_device")

    def sensitivity_device(self, rho_ptr, u_ptr, dc_ptr, p=3.0, e0=1.0, emin=1e-9):
        self.check(self.lib.hx_sensitivity_device(self.h, C.c_void_p(rho_ptr), C.c_void_p(u_ptr),
                                                  p, e0, emin, C.c_void_p(dc_ptr)),
                   "hx_sensitivity_device")

    def compliance_device(self, f_ptr, u_ptr):
        c = C.c_double()
        self.check(self.lib.hx_compliance_device(self.h, C.c_void_p(f_ptr), C.c_void_p(u_ptr),
                                                 C.byref(c)), "hx_compliance_device")
        return c.value

    def oc_update_device(self, x_ptr, dc_ptr, xnew_ptr, volfrac, move, dv_ptr=None):
        lam, steps = C.c_double(), C.c_int32()
        self.check(self.lib.hx_oc_update_device(self.h, C.c_void_p(x_ptr), C.c_void_p(dc_ptr),
                                                C.c_void_p(dv_ptr or 0), float(volfrac),
                                                float(move), C.c_void_p(xnew_ptr),
                                                C.byref(lam), C.byref(steps)),
                   "hx_oc_update_device")
        return lam.value, steps.value

    def stress_pnorm(self, u, density, E, nu, P=8.0):
        """(sigma_PN, max von Mises) of displacement u (host array)."""
        u = np.ascontiguousarray(u)
        density = np.ascontiguousarray(density, dtype=u.dtype)
        pn, vmax = C.c_double(), C.c_double()
        self.check(self.lib.hx_stress_pnorm(self.h, _dtype_code(u), _ptr(u), _ptr(density), E, nu,
                                            float(P), C.byref(pn), C.byref(vmax)),
                   "hx_stress_pnorm")
        return pn.value, vmax.value

    def compliance(self, f, u):
        f = np.ascontiguousarray(f)
        u = np.ascontiguousarray(u, dtype=f.dtype)
        c = C.c_double()
        self.check(self.lib.hx_compliance(self.h, _dtype_code(f), _ptr(f), _ptr(u), C.byref(c)),
                   "hx_compliance")
        return c.value

    def element_energy(self, u, n_elem):
        u = np.ascontiguousarray(u)
        ce = np.empty(n_elem, u.dtype)
        self.check(self.lib.hx_element_energy(self.h, _dtype_code(u), _ptr(u), _ptr(ce)),
                   "hx_element_energy")
        return ce

    def oc_update(self, x, dc, dv, volfrac, move):
        x = np.ascontiguousarray(x)
        dc = np.ascontiguousarray(dc, dtype=x.dtype)
        dv = np.ascontiguousarray(dv, dtype=x.dtype)
        xn = np.empty_like(x)
        lam = C.c_double()
        steps = C.c_int32()
        self.check(self.lib.hx_oc_update(self.h, _dtype_code(x), _ptr(x), _ptr(dc), _ptr(dv),
                                         float(volfrac), float(move), _ptr(xn), C.byref(lam),
                                         C.byref(steps)), "hx_oc_update")
        return xn, lam.value, steps.value
