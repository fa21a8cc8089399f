"""Synthetic workloads of the measured configurations (seeded, no datasets).

cantilever(nx, ny, nz): the 3D cantilever -- face x=0 fully clamped, a unit
  downward (-y, the reference's gravity direction, src/Core/Boundary.jl:329)
  load spread evenly over the nodes of the line x=nx, z=nz/2.  Location specs
  use absolute coordinates > 1 so the fraction rule of Boundary.jl:119-120
  does not apply.
random_density(...): i.i.d. U[0,1) per element from splitmix64(seed, e),
  smoothed by the Helmholtz filter (radius in element lengths, geometric
  element), affinely mapped to [rho_min, 1]; SIMP factor
  E_min + rho^p (E0 - E_min).
mbb_half_beam(nx, ny, nz): the MBB half-beam -- symmetry u_x=0 on x=0, roller
  u_y=0 on the line x=nx, y=0, unit downward load on the line x=0, y=ny.
"""
import numpy as np

from . import boundary, mesh

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64_uniform(seed, n, offset=0):
    """U[0,1) doubles: splitmix64 of (seed + 0x9E3779B97F4A7C15*(index+1)),
    top 53 bits.  The same counter-based generator is used by the oracle's
    fixture script, so inputs are reproducible element by element."""
    with np.errstate(over="ignore"):
        idx = np.arange(offset, offset + n, dtype=np.uint64) + np.uint64(1)
        z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * idx
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def simp(rho, p=3.0, e0=1.0, emin=1e-9):
    return emin + np.power(rho, p) * (e0 - emin)


def lattice_nodes(nx, ny, nz):
    """Node coordinates of generate_mesh (unit spacing) without the elements."""
    k, j, i = np.meshgrid(np.arange(nz + 1, dtype=np.float32), np.arange(ny + 1, dtype=np.float32),
                          np.arange(nx + 1, dtype=np.float32), indexing="ij")
    return np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)


def cantilever(nx, ny, nz, load=1.0, with_elements=True):
    if with_elements:
        nodes, elements, dims = mesh.generate_mesh(nx, ny, nz)
    else:
        nodes, elements = lattice_nodes(nx, ny, nz), None
    bc = boundary.get_bc_indicator(nodes.shape[0], nodes,
                                   [{"location": [0, ":", ":"], "DoFs": [1, 2, 3]}])
    f = np.zeros(3 * nodes.shape[0], np.float64)
    zline = float(nz // 2)
    if zline <= 1.0:  # keep the absolute-coordinate reading of the spec
        sel = np.nonzero((np.abs(nodes[:, 0] - nx) < 1e-4) & (np.abs(nodes[:, 2] - zline) < 1e-4))[0]
        f[3 * sel + 1] -= load / len(sel)
    else:
        boundary.apply_external_forces(f, [{"location": [nx, ":", zline], "F": [0.0, -load, 0.0]}],
                                       nodes)
    return nodes, elements, bc, f


def mbb_half_beam(nx, ny, nz, load=1.0, with_elements=True):
    if with_elements:
        nodes, elements, dims = mesh.generate_mesh(nx, ny, nz)
    else:
        nodes, elements = lattice_nodes(nx, ny, nz), None
    n = nodes.shape[0]
    bc = np.zeros((n, 3), np.float32)
    bc[np.abs(nodes[:, 0]) < 1e-4, 0] = 1.0
    bc[(np.abs(nodes[:, 0] - nx) < 1e-4) & (np.abs(nodes[:, 1]) < 1e-4), 1] = 1.0
    f = np.zeros(3 * n, np.float64)
    sel = np.nonzero((np.abs(nodes[:, 0]) < 1e-4) & (np.abs(nodes[:, 1] - ny) < 1e-4))[0]
    f[3 * sel + 1] -= load / len(sel)
    return nodes, elements, bc, f


def raw_density(n_elem, seed):
    return splitmix64_uniform(seed, n_elem)


def map_density(rho_f, rho_min=1e-3):
    lo, hi = float(rho_f.min()), float(rho_f.max())
    return rho_min + (rho_f - lo) / (hi - lo) * (1.0 - rho_min)


SEED_C1 = 20251209
