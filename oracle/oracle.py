"""ctypes wrapper of the C oracle (hexat_oracle.c) plus the OC loop restated
in numpy.  TEST INFRASTRUCTURE ONLY (see hexat_oracle.c header): the product
never imports this module.  Parity unpinned (the reference has no golden
vectors); pinned instead against scipy and analytic properties in tests/.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libhexat_oracle.so")
_lib = None


def build():
    src = os.path.join(HERE, "hexat_oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        d, i32, i64, vp = C.c_double, C.c_int32, C.c_int64, C.c_void_p
        sig = {
            "hxo_canonical_ke": (None, [d, d, d, d, vp]),
            "hxo_scalar_ke_me": (None, [d, d, d, C.c_int, vp, vp]),
            "hxo_apply_stiffness": (None, [i64, i64, vp, vp, vp, vp, vp, C.c_int]),
            "hxo_diagonal": (None, [i64, i64, vp, vp, vp, vp]),
            "hxo_cg_solve": (C.c_int, [i64, i64, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, d, d,
                                       C.c_int, C.c_int, C.POINTER(d), C.POINTER(d)]),
            "hxo_helmholtz_filter": (C.c_int, [i64, i64, vp, d, d, d, d, C.c_int, vp, vp, d,
                                               C.c_int, C.POINTER(d)]),
            "hxo_sym3_eigen": (None, [vp, vp, vp]),
            "hxo_stress": (None, [i64, i64, vp, vp, vp, d, d, vp, vp, vp, vp, vp, vp]),
            "hxo_element_energy": (None, [i64, vp, vp, vp, vp]),
            "hxo_oc_update": (C.c_int, [i64, vp, vp, vp, d, d, vp, C.POINTER(d)]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def canonical_ke(dx=1.0, dy=1.0, dz=1.0, nu=0.3):
    ke = np.zeros(576)
    lib().hxo_canonical_ke(dx, dy, dz, nu, _p(ke))
    return ke.reshape(24, 24)


def scalar_ke_me(dx=1.0, dy=1.0, dz=1.0, ref_compat=1):
    ke = np.zeros(64)
    me = np.zeros(64)
    lib().hxo_scalar_ke_me(dx, dy, dz, int(ref_compat), _p(ke), _p(me))
    return ke.reshape(8, 8), me.reshape(8, 8)


def apply_stiffness(conn0, n_nodes, ke, factor, x, nthreads=0):
    conn0 = _c(conn0, np.int32)
    ke = _c(ke, np.float64)
    factor = _c(factor, np.float64)
    x = _c(x, np.float64)
    y = np.zeros(3 * n_nodes)
    lib().hxo_apply_stiffness(n_nodes, conn0.shape[0], _p(conn0), _p(ke), _p(factor), _p(x),
                              _p(y), int(nthreads))
    return y


def diagonal(conn0, n_nodes, ke, factor):
    conn0 = _c(conn0, np.int32)
    d = np.zeros(3 * n_nodes)
    lib().hxo_diagonal(n_nodes, conn0.shape[0], _p(conn0), _p(_c(ke, np.float64)),
                       _p(_c(factor, np.float64)), _p(d))
    return d


def free_mask_from(bc_indicator, diag):
    """Free DOFs: not fixed by the BC indicator and carrying stiffness."""
    fixed = (np.asarray(bc_indicator) > 0).reshape(-1)
    return (~fixed & (diag > 0)).astype(np.uint8)


def cg_solve(conn0, n_nodes, ke, factor, free_mask, f, x0=None, max_iter=40000, tol=1e-6,
             shift_factor=0.0, precond_add=True, nthreads=0):
    """Returns (x_full, iterations, rel_res, shift); iterations -1 = breakdown."""
    conn0 = _c(conn0, np.int32)
    x = np.zeros(3 * n_nodes) if x0 is None else _c(x0, np.float64).copy()
    rel = C.c_double()
    sh = C.c_double()
    it = lib().hxo_cg_solve(n_nodes, conn0.shape[0], _p(conn0), _p(_c(ke, np.float64)),
                            _p(_c(factor, np.float64)), _p(_c(free_mask, np.uint8)),
                            _p(_c(f, np.float64)), _p(x), int(x0 is not None), int(max_iter),
                            float(tol), float(shift_factor), int(bool(precond_add)),
                            int(nthreads), C.byref(rel), C.byref(sh))
    return x, it, rel.value, sh.value


def helmholtz_filter(conn0, n_nodes, rho, dx, dy, dz, radius, ref_compat=1, tol=1e-5,
                     max_iter=200):
    conn0 = _c(conn0, np.int32)
    rho = _c(rho, np.float64)
    out = np.zeros_like(rho)
    rel = C.c_double()
    it = lib().hxo_helmholtz_filter(n_nodes, conn0.shape[0], _p(conn0), dx, dy, dz, radius,
                                    int(ref_compat), _p(rho), _p(out), tol, int(max_iter),
                                    C.byref(rel))
    return out, it, rel.value


def sym3_eigen(s6):
    s6 = _c(s6, np.float64)
    ev = np.zeros(3)
    v0 = np.zeros(3)
    lib().hxo_sym3_eigen(_p(s6), _p(ev), _p(v0))
    return ev, v0


def stress(conn0, nodes, u, E, nu, density):
    conn0 = _c(conn0, np.int32)
    ne = conn0.shape[0]
    nodes = _c(nodes, np.float64)
    out = [np.zeros((ne, 3)), np.zeros(ne), np.zeros((ne, 6)), np.zeros(ne), np.zeros((ne, 3))]
    lib().hxo_stress(nodes.shape[0], ne, _p(conn0), _p(nodes), _p(_c(u, np.float64)), E, nu,
                     _p(_c(density, np.float64)), *[_p(o) for o in out])
    return tuple(out)


def stress_pnorm(conn0, nodes, u, E, nu, density, P=8.0):
    """p-norm aggregate of the element von Mises stresses (the published
    aggregation of stress-constrained topology optimisation; no reference
    counterpart): (sum_e vm_e^P)^(1/P) = m (sum (vm_e / m)^P)^(1/P), m = max vm.
    Returns (pnorm, m)."""
    vm = stress(conn0, nodes, u, E, nu, density)[1]
    m = float(vm.max())
    if m <= 0.0:
        return 0.0, m
    return m * float(np.sum((vm / m) ** P)) ** (1.0 / P), m


def element_energy(conn0, ke, u):
    conn0 = _c(conn0, np.int32)
    ce = np.zeros(conn0.shape[0])
    lib().hxo_element_energy(conn0.shape[0], _p(conn0), _p(_c(ke, np.float64)),
                             _p(_c(u, np.float64)), _p(ce))
    return ce


def oc_update(x, dc, dv, volfrac, move):
    x = _c(x, np.float64)
    xn = np.zeros_like(x)
    lam = C.c_double()
    steps = lib().hxo_oc_update(x.shape[0], _p(x), _p(_c(dc, np.float64)),
                                _p(_c(dv, np.float64)), volfrac, move, _p(xn), C.byref(lam))
    return xn, lam.value, steps


def topopt_oc_loop(conn0, n_nodes, dims, bc_indicator, f, volfrac, radius, n_iter, p=3.0,
                   e0=1.0, emin=1e-9, nu=0.3, move=0.2, tol=1e-6, ref_compat=0,
                   filter_tol=1e-5, filter_max_iter=200, nthreads=0):
    """The OC loop (published method, no reference counterpart), restated with
    the oracle's primitives in the order the library's driver uses:
    rho = F(x); factor = SIMP(rho); warm-started PCG; c = f.u;
    dc = -p rho^(p-1) (E0-Emin) ce; dc_x = F(dc); OC bisection on x.
    Returns (compliance history, final x, final rho)."""
    ke = canonical_ke(1.0, 1.0, 1.0, nu)
    ne = conn0.shape[0]
    x = np.full(ne, volfrac)
    u = None
    hist = []
    rho = x
    for _ in range(n_iter):
        rho, _, _ = helmholtz_filter(conn0, n_nodes, x, 1.0, 1.0, 1.0, radius, ref_compat,
                                     filter_tol, filter_max_iter)
        fac = emin + np.power(np.clip(rho, 0.0, None), p) * (e0 - emin)
        diag = diagonal(conn0, n_nodes, ke, fac)
        free = free_mask_from(bc_indicator, diag)
        u, it, rel, _ = cg_solve(conn0, n_nodes, ke, fac, free, f * free, x0=u, tol=tol,
                                 nthreads=nthreads)
        c = float(np.dot(f, u))
        hist.append(c)
        ce = element_energy(conn0, ke, u)
        dc = -p * np.power(np.clip(rho, 0.0, None), p - 1) * (e0 - emin) * ce
        dcf, _, _ = helmholtz_filter(conn0, n_nodes, dc, 1.0, 1.0, 1.0, radius, ref_compat,
                                     filter_tol, filter_max_iter)
        x, _, _ = oc_update(x, dcf, np.ones(ne), volfrac, move)
    return np.array(hist), x, rho


def structured_conn0(nx, ny, nz):
    """0-based Hex8 connectivity of generate_mesh (src/Mesh/Mesh.jl:44-55):
    element e = i + nx*(j + ny*k), corners in NAT_COORDS order."""
    nnx, nny = nx + 1, ny + 1
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    n0 = (i + nnx * (j + nny * k)).ravel()
    off = [0, 1, 1 + nnx, nnx, nnx * nny, 1 + nnx * nny, 1 + nnx + nnx * nny, nnx + nnx * nny]
    return (n0[:, None] + np.array(off)[None, :]).astype(np.int32)


def radius_schedule(it, n_iter, h, max_domain_dim, R_init_perc=0.0, R_interm_perc=0.0,
                    R_final_perc=0.0, R_interm_iter_perc=50.0):
    """Filter radius of update_density!, src/Optimization/TopOpt.jl:216-255,
    with Julia's types: the percentages and element sizes are Float32,
    max_domain_dim is taken as Float64 (a YAML number), so the lengths are
    Float64; t, the guard 1.2 * mean element size and the divisor 2.5 are
    Float32.  Returns (R_length, R_effective) as Python floats."""
    f32 = np.float32
    dx, dy, dz = (f32(v) for v in h)
    avg = (dx + dy + dz) / f32(3.0)
    ri = f32(R_init_perc) / f32(100.0)
    rm = f32(R_interm_perc) / f32(100.0)
    rf = f32(R_final_perc) / f32(100.0)
    rip = f32(R_interm_iter_perc) / f32(100.0)
    Ri, Rm, Rf = (float(v) * float(max_domain_dim) for v in (ri, rm, rf))
    iter_interm = max(1, int(np.rint(rip * f32(n_iter))))
    calc = min(it, n_iter)
    if calc <= iter_interm:
        t = f32(calc - 1) / f32(iter_interm - 1) if iter_interm > 1 else f32(0.0)
        R = Ri * float(f32(1.0) - t) + Rm * float(t)
    else:
        t = (f32(calc - iter_interm) / f32(n_iter - iter_interm)) if n_iter > iter_interm \
            else f32(0.0)
        R = Rm * float(f32(1.0) - t) + Rf * float(t)
    safe = f32(1.2) * avg
    if R < float(safe):
        return float(safe), float(safe / f32(2.5))
    return R, R / 2.5


def update_density(density, l1, protected, E, allowable, it, n_iter, original, min_d, max_d,
                   dims, h, max_domain_dim, filter_tol=1e-5, stress_regularization_ratio=0.0,
                   R_init_perc=0.0, R_interm_perc=0.0, R_final_perc=0.0,
                   R_interm_iter_perc=50.0, final_density_threshold=0.95,
                   max_culling_ratio=0.1, filtered=None):
    """Restatement of TopologyOptimization.update_density!
    (src/Optimization/TopOpt.jl:139-405) in float32 numpy on the structured
    grid `dims` (elements in grid order):
      * optional stress regularisation: the L1 stress field filtered with
        radius ratio * mean element size (:176-211);
      * radius schedule and guard (:216-255, radius_schedule);
      * stress-ratio proposal clamp((l1 / allowable) / E, min, max), the
        original density on protected elements (:260-271);
      * Helmholtz filter of the proposal with the reference element
        (ref_compat, GPUHelmholtz.apply_gpu_filter! at :286), radius rounded
        to Float32 as the filter workspace does, at most 200 iterations;
      * clamp and the largest change over unprotected elements (:327-343);
      * culling below threshold * iter / n_iter (the final threshold once iter
        exceeds n_iter), at most floor(active * max_culling_ratio) elements,
        the weakest first, ties in element order (:350-395; Julia's default
        sort is stable);
      * protected elements re-enforced (:398-402).
    `filtered` (float32), when given, replaces the filter's output, so the
    rest can be compared bit for bit with a device run that reports its
    filtered field.  Returns (density, l1, (max_change, R_length,
    threshold, filter_iters, filter_res), filtered)."""
    f32 = np.float32
    nx, ny, nz = dims
    dens = np.array(density, dtype=f32)
    l1 = np.array(l1, dtype=f32)
    orig = np.asarray(original, dtype=f32)
    prot = np.asarray(protected, dtype=bool)
    min_d, max_d, E, allowable = f32(min_d), f32(max_d), f32(E), f32(allowable)
    conn0 = None
    dxf, dyf, dzf = (f32(v) for v in h)
    avg = (dxf + dyf + dzf) / f32(3.0)
    nn = (nx + 1) * (ny + 1) * (nz + 1)
    ratio = f32(stress_regularization_ratio)
    if ratio > 1e-6:
        conn0 = structured_conn0(nx, ny, nz)
        r = float(f32(ratio * avg))
        s, _, _ = helmholtz_filter(conn0, nn, l1.astype(np.float64), float(dxf), float(dyf),
                                   float(dzf), r, 1, float(f32(filter_tol)), 200)
        l1 = s.astype(f32)
    R_length, R_eff = radius_schedule(it, n_iter, h, max_domain_dim, R_init_perc, R_interm_perc,
                                      R_final_perc, R_interm_iter_perc)
    with np.errstate(divide="ignore", invalid="ignore"):
        val = (l1 / allowable) / E
    prop = np.where(prot, orig, np.clip(val, min_d, max_d)).astype(f32)
    iters, res = 0, 0.0
    if filtered is None:
        if conn0 is None:
            conn0 = structured_conn0(nx, ny, nz)
        fo, iters, res = helmholtz_filter(conn0, nn, prop.astype(np.float64), float(dxf),
                                          float(dyf), float(dzf), float(f32(R_eff)), 1,
                                          float(f32(filter_tol)), 200)
        filtered = fo.astype(f32)
    filtered = np.asarray(filtered, dtype=f32)
    new = np.clip(filtered, min_d, max_d).astype(f32)
    change = np.abs(new - dens)
    max_change = float(change[~prot].max()) if np.any(~prot) else 0.0
    dens = np.where(prot, dens, new)
    thr = f32(final_density_threshold) if it > n_iter else \
        f32(final_density_threshold) * (f32(it) / f32(n_iter))
    active = int(np.count_nonzero(~prot & (dens > min_d)) + np.count_nonzero(prot & (orig > min_d)))
    cand = np.nonzero(~prot & (dens > min_d) & (dens < thr))[0]
    max_allowed = int(np.floor(f32(active) * f32(max_culling_ratio)))
    if cand.size > max_allowed:
        order = np.argsort(dens[cand], kind="stable")
        cand = cand[order[:max_allowed]]
    dens[cand] = min_d
    dens[prot] = orig[prot]
    return dens, l1, (max_change, R_length, float(thr), iters, res), filtered


def webdata_arrays(dims, h, density, l1, principal, threshold):
    """Restatement of export_binary_for_web's arrays
    (src/IO/Postprocessing.jl:172-193) on generate_mesh's grid, in float32:
    findall(density .>= threshold) in element order; centroid = Float32 sum
    of the 8 corner coordinates (Int * Float32 products) in NAT_COORDS order
    times 0.125f0 (MeshUtilities.element_centroid); L1 stress times the sign
    of the principal stress of largest magnitude.  Returns (centroids (n, 3),
    densities, signed L1)."""
    f32 = np.float32
    nx, ny, nz = dims
    d = np.asarray(density, f32)
    idx = np.nonzero(d >= f32(threshold))[0]
    i = idx % nx
    j = (idx // nx) % ny
    k = idx // (nx * ny)
    cent = np.zeros((idx.size, 3), f32)
    corner = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1),
              (0, 1, 1)]
    for a, (ijk, hh) in enumerate(zip((i, j, k), h)):
        acc = np.zeros(idx.size, f32)
        for c in corner:
            acc = (acc + (ijk + c[a]).astype(f32) * f32(hh)).astype(f32)
        cent[:, a] = acc * f32(0.125)
    pr = np.asarray(principal, f32).reshape(-1, 3)[idx]
    sgn = np.sign(pr[:, 0])
    amax = np.abs(pr[:, 0])
    for c in (1, 2):
        big = np.abs(pr[:, c]) > amax
        amax = np.where(big, np.abs(pr[:, c]), amax)
        sgn = np.where(big, np.sign(pr[:, c]), sgn)
    sl1 = (np.asarray(l1, f32)[idx] * sgn.astype(f32)).astype(f32)
    return cent, d[idx], sl1
