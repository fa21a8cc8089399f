"""Structured Hex8 mesh in the reference's layout (src/Mesh/Mesh.jl:13-60).

Nodes are numbered i fastest, then j, then k (Mesh.jl:13-15); element
corners follow NAT_COORDS (src/Core/Element.jl:8-17).  Arrays mirror the
Julia ones: `nodes` is (nN, 3) float32, `elements` is (nE, 8) int64 and
1-based.
"""
import numpy as np


def node_index(i, j, k, nnx, nny):
    """1-based node index of 1-based lattice position (Mesh.jl:13-15)."""
    return i + (j - 1) * nnx + (k - 1) * nnx * nny


def generate_mesh(nelem_x, nelem_y, nelem_z, dx=1.0, dy=1.0, dz=1.0):
    """generate_mesh (Mesh.jl:23-60): returns (nodes, elements, dims)."""
    nnx, nny, nnz = nelem_x + 1, nelem_y + 1, nelem_z + 1
    k, j, i = np.meshgrid(np.arange(nnz), np.arange(nny), np.arange(nnx), indexing="ij")
    nodes = np.stack([i.ravel() * np.float32(dx), j.ravel() * np.float32(dy),
                      k.ravel() * np.float32(dz)], axis=1).astype(np.float32)
    ek, ej, ei = np.meshgrid(np.arange(nelem_z), np.arange(nelem_y), np.arange(nelem_x),
                             indexing="ij")
    n1 = (ei + ej * nnx + ek * nnx * nny).ravel().astype(np.int64) + 1
    px, py = 1, nnx
    pz = nnx * nny
    elements = np.stack([n1, n1 + px, n1 + px + py, n1 + py,
                         n1 + pz, n1 + px + pz, n1 + px + py + pz, n1 + py + pz], axis=1)
    return nodes, elements, (nnx, nny, nnz)


def connectivity0(elements):
    """0-based int32 row-major (nE, 8) copy of a Julia-layout element array."""
    return np.ascontiguousarray(elements - 1, dtype=np.int32)
