"""Independent numpy restatements used to pin the oracle and the library."""
import numpy as np
import scipy.sparse as sp

NAT = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]


def haar_ke(h, nu):
    """Ke of a box from exact 1D integrals (Kronecker closed form), unit E:
    K_ij = lam int dNa/dxi dNb/dxj + mu int dNa/dxj dNb/dxi + mu delta_ij int grad.grad."""
    lam = nu / ((1 + nu) * (1 - 2 * nu))
    mu = 1 / (2 * (1 + nu))
    S = [np.array([[1, -1], [-1, 1]]) / ha for ha in h]
    M = [np.array([[2, 1], [1, 2]]) * ha / 6 for ha in h]
    Cm = np.array([[-0.5, -0.5], [0.5, 0.5]])      # int N'_a N_b
    CT = Cm.T                                        # int N_a N'_b

    def op(i, j):  # int d_i N_A d_j N_B as an 8x8 in NAT corner order
        out = np.zeros((8, 8))
        for A, a in enumerate(NAT):
            for B, b in enumerate(NAT):
                v = 1.0
                for ax in range(3):
                    if ax == i and ax == j:
                        v *= S[ax][a[ax], b[ax]]
                    elif ax == i:
                        v *= Cm[a[ax], b[ax]]
                    elif ax == j:
                        v *= CT[a[ax], b[ax]]
                    else:
                        v *= M[ax][a[ax], b[ax]]
                out[A, B] = v
        return out
    K = np.zeros((24, 24))
    lap = sum(op(k, k) for k in range(3))
    for i in range(3):
        for j in range(3):
            blk = lam * op(i, j) + mu * op(j, i) + (mu * lap if i == j else 0)
            K[i::3, j::3] = blk
    return K


def rigid_modes(h):
    X = np.array([[(a[0] - 0.5) * h[0], (a[1] - 0.5) * h[1], (a[2] - 0.5) * h[2]] for a in NAT])
    R = np.zeros((24, 6))
    for n in range(8):
        x, y, z = X[n]
        R[3 * n:3 * n + 3, 0:3] = np.eye(3)
        R[3 * n:3 * n + 3, 3] = [-y, x, 0]
        R[3 * n:3 * n + 3, 4] = [0, -z, y]
        R[3 * n:3 * n + 3, 5] = [z, 0, -x]
    return R


def assemble(conn0, n_nodes, ke, factor):
    """Sparse assembled K = sum_e factor_e Ke (CSR)."""
    ne = conn0.shape[0]
    dofs = (3 * conn0[:, :, None] + np.arange(3)[None, None, :]).reshape(ne, 24)
    rows = np.repeat(dofs, 24, axis=1).ravel()
    cols = np.tile(dofs, (1, 24)).ravel()
    vals = (factor[:, None, None] * ke[None]).reshape(ne, 576).ravel()
    return sp.csr_matrix((vals, (rows, cols)), shape=(3 * n_nodes, 3 * n_nodes))


def prune_system(nodes, elements, density, threshold, bc, F):
    """numpy restatement of MeshPruner.prune_system (src/Mesh/MeshPruner.jl:18-112):
    keeps elements with density > threshold and the nodes they use, renumbered
    in original order.  Returns (nodes, elements(1-based), bc, F, density,
    new_to_old (0-based))."""
    active = np.nonzero(density > threshold)[0]
    used = np.zeros(nodes.shape[0], bool)
    used[elements[active].ravel() - 1] = True
    new_to_old = np.nonzero(used)[0]
    old_to_new = np.full(nodes.shape[0], -1, np.int64)
    old_to_new[new_to_old] = np.arange(len(new_to_old))
    el = old_to_new[elements[active] - 1] + 1
    Fr = F.reshape(-1, 3)[new_to_old].reshape(-1)
    return nodes[new_to_old], el, bc[new_to_old], Fr, density[active], new_to_old


def reconstruct_full_solution(u_red, new_to_old, n_full):
    """MeshPruner.reconstruct_full_solution (MeshPruner.jl:120-138)."""
    u = np.zeros((n_full, 3), u_red.dtype)
    u[new_to_old] = u_red.reshape(-1, 3)
    return u.reshape(-1)


def free_dofs(conn0, n_nodes, factor, bc_indicator):
    """Free-DOF mask as the library forms it: not fixed by the BC indicator
    and the node carries stiffness (sum of its elements' factors > 0)."""
    s = np.zeros(n_nodes)
    np.add.at(s, conn0.ravel(), np.repeat(factor, 8))
    fixed = (np.asarray(bc_indicator) > 0).reshape(-1)
    return (~fixed & np.repeat(s > 0, 3)).astype(np.float64)


def gpu_solver_reference(K, free, f, tol, max_iter, shift_factor, ref_retry=True,
                         divergence_checks=True, keep_best=True, u0=None):
    """numpy restatement of the reference GPU solver's attempt loop,
    src/Solvers/GPUSolver.jl:380-606, on an assembled K (scipy CSR) restricted
    to the free DOFs by the 0/1 mask `free`, with the library's documented
    deviations: breakdown is !(p.Ap > 0) (the reference tests |p.Ap| < 1e-20)
    and there is no AMG preconditioner to switch to.

    Per attempt (at most 3 with ref_retry): shift s = factor * max diag over
    free DOFs; M^-1 = 1 / (diag + s); x from u0 on attempt 1, else 0; Jacobi-
    PCG with the divergence tests in the reference's order (100x over the
    attempt's best after 50 iterations; NaN/Inf; > 1000 ||b||); the best
    iterate is snapshotted only while its residual is below 1e-2 (the
    snapshot starts as the attempt's initial x).  After a failed attempt:
    diverged or best > 0.1 -> factor x 10; best < 5e-2 -> accept the snapshot
    ("acceptable stagnation"); otherwise keep it as the global best when it
    is the lowest so far and factor x 5.  When every attempt fails the global
    best (zeros if none) is returned.

    Returns a dict: u, status ('converged', 'stalled', 'failed'), attempts,
    shift (of the last attempt), reason of the last attempt ('converged',
    'breakdown', 'diverged', 'nonfinite', 'maxiter'), best (last attempt's
    best relative residual), iterations (all attempts)."""
    n = K.shape[0]
    diag = K.diagonal()
    maxd = float(np.max(diag[free > 0])) if np.any(free > 0) else 0.0
    b = f * free
    bnorm = float(np.linalg.norm(b))
    factor = shift_factor
    attempts = 3 if ref_retry else 1
    global_best, global_low = None, np.inf
    total = 0
    out = None
    for attempt in range(1, attempts + 1):
        s = factor * maxd
        minv = np.where(free > 0, 1.0 / (diag + s), 0.0)
        x = (u0 * free).copy() if (u0 is not None and attempt == 1) else np.zeros(n)
        A = lambda v: (K @ (v * free) + s * v) * free
        r = b - A(x)
        z = minv * r
        p = z.copy()
        rz = float(r @ z)
        best, snap = np.inf, x.copy()
        reason = "maxiter"
        it = 0
        if bnorm == 0.0:
            return {"u": np.zeros(n), "status": "converged", "attempts": attempt, "shift": s,
                    "reason": "zero_rhs", "best": 0.0, "iterations": 0}
        # a non-finite initial residual ends the attempt before its first
        # iteration (the reference meets the same failure one step later, as
        # a NaN denominator)
        if not np.isfinite(float(np.sqrt(r @ r)) / bnorm):
            reason, it = "nonfinite", 0
            max_iter_eff = 0
        else:
            max_iter_eff = max_iter
        for it in range(1, max_iter_eff + 1):
            q = A(p)
            pq = float(p @ q)
            if not (pq > 0.0):
                reason = "breakdown"
                break
            alpha = rz / pq
            x = x + alpha * p
            r = r - alpha * q
            rel = float(np.sqrt(r @ r)) / bnorm
            if divergence_checks and it > 50 and rel > 100.0 * best:
                reason = "diverged"
                break
            if not np.isfinite(rel):
                reason = "nonfinite"
                break
            if divergence_checks and rel > 1000.0:
                reason = "diverged"
                break
            if rel < best:
                best = rel
                if keep_best and rel < 1e-2:
                    snap = x.copy()
            if rel < tol:
                reason = "converged"
                break
            z = minv * r
            rzn = float(r @ z)
            p = z + (rzn / rz) * p
            rz = rzn
        total += it if max_iter_eff else 0
        if reason == "converged":
            return {"u": x, "status": "converged", "attempts": attempt, "shift": s,
                    "reason": reason, "best": best, "iterations": total}
        out = {"attempts": attempt, "shift": s, "reason": reason, "best": best,
               "iterations": total}
        if not ref_retry:
            out.update(u=x, status="failed")
            return out
        failed_badly = reason in ("breakdown", "diverged", "nonfinite") or best > 0.1
        if not failed_badly and best < 5e-2:
            out.update(u=snap if keep_best else x, status="stalled")
            return out
        if failed_badly:
            factor *= 10.0
        else:
            if best < global_low and keep_best:
                global_low, global_best = best, snap.copy()
            factor *= 5.0
    out.update(u=global_best if global_best is not None else np.zeros(n), status="failed")
    return out
