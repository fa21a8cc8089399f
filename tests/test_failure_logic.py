"""(CPU) The numpy restatement of the reference solver's attempt loop
(tests.helpers.gpu_solver_reference, src/Solvers/GPUSolver.jl:380-606) on the
inputs the GPU failure-handling tests use: every decision those tests rely
on, with its margin, so a change that moves one near its threshold fails
here, on the CPU, first."""
import numpy as np

from tests.helpers import assemble, free_dofs, gpu_solver_reference, haar_ke

DIMS = (10, 4, 4)


def _problem(hx, seed=3, negative=0.0):
    nodes, el, bc, f = hx.workloads.cantilever(*DIMS)
    c0 = hx.mesh.connectivity0(el)
    rng = np.random.default_rng(seed)
    fac = hx.workloads.simp(rng.uniform(0.2, 1.0, c0.shape[0]))
    if negative:
        fac[rng.uniform(size=fac.shape) < 0.15] = -negative
    K = assemble(c0, nodes.shape[0], haar_ke((1.0, 1.0, 1.0), 0.3), fac)
    return f, K, free_dofs(c0, nodes.shape[0], fac, bc)


def test_stagnation_bands(hx):
    f, K, free = _problem(hx)
    r = gpu_solver_reference(K, free, f, 1e-12, 135, 1e-9)
    assert r["status"] == "stalled" and r["attempts"] == 1 and 2e-3 < r["best"] < 8e-3
    assert np.any(r["u"] != 0)
    r = gpu_solver_reference(K, free, f, 1e-12, 127, 1e-9)
    assert r["status"] == "stalled" and 1.5e-2 < r["best"] < 4.5e-2 and np.all(r["u"] == 0)
    r = gpu_solver_reference(K, free, f, 1e-12, 110, 1e-9)
    assert r["status"] == "failed" and r["attempts"] == 3 and 5.5e-2 < r["best"] < 9e-2
    maxd = K.diagonal()[free > 0].max()
    assert abs(r["shift"] - 1e-9 * 25.0 * maxd) <= 1e-12 * r["shift"] and np.all(r["u"] == 0)


def test_hard_failures(hx):
    f, K, free = _problem(hx)
    fn = f.copy()
    fn[np.nonzero(free)[0][7]] = np.nan
    r = gpu_solver_reference(K, free, fn, 1e-8, 500, 1e-6)
    assert r["status"] == "failed" and r["attempts"] == 3 and r["reason"] == "nonfinite"
    u0 = np.random.default_rng(2).standard_normal(f.shape[0]) * 1e6
    r = gpu_solver_reference(K, free, f, 1e-8, 3000, 1e-9, u0=u0)
    assert r["status"] == "converged" and r["attempts"] == 2
    f, K, free = _problem(hx, seed=1, negative=0.3)
    idx = np.nonzero(free)[0]
    lo = np.linalg.eigvalsh(K[idx][:, idx].toarray())[0]
    maxd = K.diagonal()[idx].max()
    assert -0.24 < lo < -0.23 and 0.89 < maxd < 0.90
    for sf, att in ((0.05, 2), (0.01, 3)):
        r = gpu_solver_reference(K, free, f, 1e-8, 2000, sf)
        assert r["status"] == "converged" and r["attempts"] == att
        assert r["shift"] > -lo * 1.5  # the converging attempt is clearly definite
    r = gpu_solver_reference(K, free, f, 1e-8, 2000, 1e-3)
    assert r["status"] == "failed" and r["attempts"] == 3 and r["shift"] < -lo * 0.5
