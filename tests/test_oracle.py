"""Pins of the CPU oracle (no GPU): analytic properties of the element
matrices, a scipy direct solve of the assembled system, the filter's
constant-field behaviour, the eigen-solver and the OC update invariants."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from tests.helpers import assemble, haar_ke, rigid_modes


@pytest.mark.parametrize("h,nu", [((1, 1, 1), 0.3), ((1.3, 0.7, 2.1), 0.25), ((0.5, 2, 1), 0.45)])
def test_ke_properties(orc, h, nu):
    ke = orc.canonical_ke(*h, nu)
    assert np.abs(ke - ke.T).max() < 1e-14 * np.abs(ke).max()
    assert np.linalg.matrix_rank(ke, tol=1e-10 * np.abs(ke).max()) == 18
    w = np.linalg.eigvalsh(ke)
    assert w.min() > -1e-12 * w.max()
    # rigid-body modes (3 translations, 3 rotations) are in the null space
    R = rigid_modes(h)
    assert np.abs(ke @ R).max() < 1e-12 * np.abs(ke).max()


@pytest.mark.parametrize("h,nu", [((1, 1, 1), 0.3), ((1.3, 0.7, 2.1), 0.25)])
def test_ke_matches_independent_closed_form(orc, h, nu):
    """Gauss-quadrature Ke == Kronecker closed form (independent derivation)."""
    ke = orc.canonical_ke(*h, nu)
    assert np.abs(ke - haar_ke(h, nu)).max() < 1e-13 * np.abs(ke).max()


def test_ke_unit_cube_known_values(orc):
    ke = orc.canonical_ke(1, 1, 1, 0.3)
    # unit cube, E=1: K[0,0] = (lam+2mu) S M M + mu (M S M + M M S) = (lam + 4 mu)/9
    nu = 0.3
    lam, mu = nu / ((1 + nu) * (1 - 2 * nu)), 1 / (2 * (1 + nu))
    assert ke[0, 0] == pytest.approx((lam + 4 * mu) / 9, rel=1e-13)
    assert ke[0, 0] == pytest.approx(haar_ke((1, 1, 1), 0.3)[0, 0], rel=1e-14)


@pytest.mark.parametrize("ref_compat,scale", [(0, 1.0), (1, 1.5)])
def test_scalar_matrices(orc, ref_compat, scale):
    ke, me = orc.scalar_ke_me(1, 1, 1, ref_compat)
    assert me.sum() == pytest.approx(scale, rel=1e-13)   # the reference element is 1.5 dz tall
    assert np.abs(ke.sum(1)).max() < 1e-13                 # constants in the null space
    if ref_compat:
        assert ke[0, 0] == pytest.approx(0.4074074074, rel=1e-8)
    else:
        assert ke[0, 0] == pytest.approx(1.0 / 3.0, rel=1e-12)


def test_apply_matches_assembled(orc, hx):
    nodes, el, _ = hx.mesh.generate_mesh(4, 3, 2)
    c0 = hx.mesh.connectivity0(el)
    rng = np.random.default_rng(1)
    fac = rng.uniform(0.1, 1, c0.shape[0])
    fac[3] = 0.0
    ke = orc.canonical_ke()
    K = assemble(c0, nodes.shape[0], ke, fac)
    x = rng.standard_normal(3 * nodes.shape[0])
    y = orc.apply_stiffness(c0, nodes.shape[0], ke, fac, x, nthreads=3)
    assert np.abs(y - K @ x).max() < 1e-12 * np.abs(K @ x).max()
    d = orc.diagonal(c0, nodes.shape[0], ke, fac)
    assert np.abs(d - K.diagonal()).max() < 1e-14


def test_cg_matches_direct_solve(orc, hx):
    nodes, el, bc, f = hx.workloads.cantilever(12, 4, 4)
    c0 = hx.mesh.connectivity0(el)
    rng = np.random.default_rng(2)
    fac = hx.workloads.simp(rng.uniform(0.05, 1, c0.shape[0]))
    ke = orc.canonical_ke()
    nN = nodes.shape[0]
    K = assemble(c0, nN, ke, fac)
    d = orc.diagonal(c0, nN, ke, fac)
    free = orc.free_mask_from(bc, d).astype(bool)
    uf = spla.spsolve(K[free][:, free].tocsc(), f[free])
    x, it, rel, _ = orc.cg_solve(c0, nN, ke, fac, free.astype(np.uint8), f * free, tol=1e-10)
    assert it > 0 and rel < 1e-10
    assert np.abs(x[free] - uf).max() < 1e-7 * np.abs(uf).max()
    assert np.all(x[~free] == 0)


def test_cg_shift_semantics(orc, hx):
    """clamp (CPUSolver.jl:170) vs additive (GPUSolver.jl:402) both solve (K+sI)u=f."""
    nodes, el, bc, f = hx.workloads.cantilever(6, 3, 3)
    c0 = hx.mesh.connectivity0(el)
    fac = np.ones(c0.shape[0])
    ke = orc.canonical_ke()
    nN = nodes.shape[0]
    K = assemble(c0, nN, ke, fac)
    d = orc.diagonal(c0, nN, ke, fac)
    free = orc.free_mask_from(bc, d).astype(bool)
    s = 1e-3 * d[free].max()
    uf = spla.spsolve((K[free][:, free] + s * sp.eye(free.sum())).tocsc(), f[free])
    for add in (True, False):
        x, it, rel, sh = orc.cg_solve(c0, nN, ke, fac, free.astype(np.uint8), f * free, tol=1e-11,
                                      shift_factor=1e-3, precond_add=add)
        assert sh == pytest.approx(s)
        assert np.abs(x[free] - uf).max() < 1e-8 * np.abs(uf).max()


def test_filter_constant_field(orc, hx):
    nodes, el, _ = hx.mesh.generate_mesh(6, 5, 4)
    c0 = hx.mesh.connectivity0(el)
    rho = np.full(c0.shape[0], 0.3)
    out0, it0, _ = orc.helmholtz_filter(c0, nodes.shape[0], rho, 1, 1, 1, 1.5, 0, tol=1e-12)
    assert np.abs(out0 - 0.3).max() < 1e-9
    # the reference element (1.5 dz tall) shrinks a constant field by 1/1.5
    out1, it1, _ = orc.helmholtz_filter(c0, nodes.shape[0], rho, 1, 1, 1, 1.5, 1, tol=1e-12)
    assert np.abs(out1 - 0.2).max() < 1e-9
    assert it0 % 10 == 0 and it1 % 10 == 0


def test_filter_matches_direct(orc, hx):
    nodes, el, _ = hx.mesh.generate_mesh(7, 5, 4)
    c0 = hx.mesh.connectivity0(el)
    nN = nodes.shape[0]
    rho = hx.workloads.splitmix64_uniform(7, c0.shape[0])
    for rc in (0, 1):
        kes, mes = orc.scalar_ke_me(1, 1, 1, rc)
        A = sp.lil_matrix((nN, nN))
        b = np.zeros(nN)
        for e in range(c0.shape[0]):
            idx = c0[e]
            A[np.ix_(idx, idx)] += 2.0 ** 2 * kes + mes
            b[idx] += rho[e] / 8
        xs = spla.spsolve(A.tocsc(), b)
        want = xs[c0].mean(1)
        got, it, rel = orc.helmholtz_filter(c0, nN, rho, 1, 1, 1, 2.0, rc, tol=1e-12,
                                            max_iter=2000)
        assert np.abs(got - want).max() < 1e-9


def test_sym3_eigen(orc):
    rng = np.random.default_rng(3)
    for _ in range(50):
        a = rng.standard_normal((3, 3))
        s = a + a.T
        s6 = np.array([s[0, 0], s[1, 1], s[2, 2], s[0, 1], s[1, 2], s[0, 2]])
        ev, v0 = orc.sym3_eigen(s6)
        w, V = np.linalg.eigh(s)
        assert np.allclose(ev, w[::-1], atol=1e-12)
        v = V[:, -1] * np.sign(V[np.argmax(np.abs(V[:, -1])), -1])
        assert np.allclose(v0, v, atol=1e-9)


def test_stress_affine_field(orc, hx):
    """A linear displacement field gives the exact uniform stress."""
    nodes, el, _ = hx.mesh.generate_mesh(3, 2, 2)
    c0 = hx.mesh.connectivity0(el)
    G = np.array([[1e-3, 2e-4, -1e-4], [3e-4, -2e-3, 5e-4], [0, 1e-4, 4e-4]])
    u = (nodes.astype(np.float64) @ G.T).reshape(-1)
    dens = np.full(c0.shape[0], 0.5)
    pr, vm, vo, l1, dr = orc.stress(c0, nodes, u, 2.0, 0.3, dens)
    eps = 0.5 * (G + G.T)
    E, nu = 2.0 * 0.5, 0.3
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    sig = lam * np.trace(eps) * np.eye(3) + 2 * mu * eps
    want = np.array([sig[0, 0], sig[1, 1], sig[2, 2], sig[0, 1], sig[1, 2], sig[0, 2]])
    assert np.abs(vo - want).max() < 1e-12
    assert np.allclose(pr[0], np.linalg.eigvalsh(sig)[::-1], atol=1e-12)
    assert np.allclose(l1, np.abs(np.linalg.eigvalsh(sig)).sum())


def test_oc_update_invariants(orc):
    rng = np.random.default_rng(4)
    n = 1000
    x = rng.uniform(0.2, 0.45, n)   # volfrac 0.3 reachable within the move limit
    dc = -rng.uniform(0.1, 2, n)
    xn, lam, steps = orc.oc_update(x, dc, np.ones(n), 0.3, 0.2)
    assert np.all(xn >= np.maximum(0, x - 0.2) - 1e-15)
    assert np.all(xn <= np.minimum(1, x + 0.2) + 1e-15)
    assert abs(xn.mean() - 0.3) < 5e-3
    assert 10 < steps < 80
