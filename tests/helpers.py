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
