"""Generates tests/golden/c0_oc_loop.npz: the C0 topology-optimisation loop
run by the CPU oracle (a restatement of the reference's solver, filter and
element; the OC update is the published method).

C0: cantilever 60x20x20 unit Hex8 elements, E0 = 1, Emin = 1e-9, nu = 0.3,
SIMP p = 3, volume fraction 0.3 from a uniform start, Helmholtz filter
radius 1.5 with the reference's element (ref_compat), 50 OC iterations with
move limit 0.2, each solve Jacobi-PCG to rtol 1e-6 warm-started from the
previous displacement.  Stored: the compliance history, the final design
variables x and the final physical densities rho.

Run from the repository root: python tests/golden/make_c0_golden.py
"""
import importlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

DIMS = (60, 20, 20)
PARAMS = dict(volfrac=0.3, radius=1.5, n_iter=50, p=3.0, e0=1.0, emin=1e-9, nu=0.3, move=0.2,
              tol=1e-6, ref_compat=1, filter_tol=1e-5, filter_max_iter=200)


def main():
    from oracle import oracle
    hx = importlib.import_module("2025_12_09_hexat_v069_b200")
    W = hx.workloads
    nodes, el, bc, f = W.cantilever(*DIMS)
    conn0 = hx.mesh.connectivity0(el)
    t0 = time.time()
    hist, x, rho = oracle.topopt_oc_loop(conn0, nodes.shape[0], DIMS, bc, f, **PARAMS)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c0_oc_loop.npz")
    np.savez_compressed(out, compliance=hist, x=x, rho=rho, dims=np.array(DIMS),
                        **{k: np.array(v) for k, v in PARAMS.items()})
    print(f"{len(hist)} iterations in {time.time() - t0:.1f} s; c: {hist[0]:.6g} -> "
          f"{hist[-1]:.6g}; wrote {out}")


if __name__ == "__main__":
    main()
