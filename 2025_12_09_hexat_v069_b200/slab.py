"""Multi-GPU solve by slab decomposition of the structured grid.

The reference solves on one GPU (src/Main.jl:179).  Here one process per
GPU owns a slab of element planes along z and the node planes bounding it;
neighbouring slabs share one node plane.  In the grid's numbering
(node n = i + NXn*(j + NYn*k)) a node plane is a contiguous run of
3*NXn*NYn values, so a slab is a contiguous range of every nodal vector and
the shared plane is exchanged straight from the vector's memory, without
packing.  (The x-slab split also fits the structured operator; z-slabs are
chosen because their halo is contiguous in this layout.)

Per Jacobi-PCG iteration (the algorithm of src/Solvers/CPUSolver.jl:150-212
and of the library's single-GPU solver):
  * q = K p on the slab's elements (the library's structured operator),
    then the shared planes are summed with the neighbours (one send/receive
    of one node plane per neighbour): K p is a sum over elements, so the
    partial sums of two slabs add up to the global product;
  * the shift s p and the free-DOF mask are applied after that sum, so both
    copies of a shared plane hold the same complete q;
  * p.q, r.z and r.r are nodal sums: each rank counts the nodes it owns (a
    shared plane belongs to the upper slab), then one all-reduce of the
    scalars per dot product.
The diagonal and the free-DOF mask are formed the same way (partial diagonal,
shared-plane sum).  Collectives go through torch.distributed (NCCL between
GPUs, gloo on CPU).

Status: the decomposition, exchange and dot products are tested with two
gloo ranks on CPU against the single-domain oracle solve; the GPU path runs
the library's operator per slab with the vector updates in torch, and is
not measured on multi-GPU hardware.
"""
import numpy as np


def split_planes(nze, world):
    """Element planes per rank, as even as possible: [(e0, e1), ...]."""
    base, extra = divmod(nze, world)
    out, e0 = [], 0
    for r in range(world):
        e1 = e0 + base + (1 if r < extra else 0)
        out.append((e0, e1))
        e0 = e1
    if any(e1 <= e0 for e0, e1 in out):
        raise ValueError(f"{nze} element planes cannot feed {world} slabs")
    return out


class Slab:
    """Geometry of rank `rank`'s slab of an nx x ny x nz element grid."""

    def __init__(self, dims, rank, world):
        self.nx, self.ny, self.nz = dims
        self.rank, self.world = rank, world
        self.e0, self.e1 = split_planes(self.nz, world)[rank]
        self.nzl = self.e1 - self.e0                       # local element planes
        self.plane = 3 * (self.nx + 1) * (self.ny + 1)     # values per node plane
        self.n = self.plane * (self.nzl + 1)               # local nodal values
        self.lower = rank > 0                              # shares its bottom plane
        self.upper = rank < world - 1                      # shares its top plane

    def elem_slice(self):
        """Global element range of the slab (elements are plane-major)."""
        pe = self.nx * self.ny
        return slice(self.e0 * pe, self.e1 * pe)

    def node_slice(self):
        """Global nodal-value range of the slab (bounding planes included)."""
        return slice(self.e0 * self.plane, (self.e1 + 1) * self.plane)

    def owned(self):
        """Local nodal-value range this rank counts in nodal dot products: its
        planes except the top one when an upper slab shares it."""
        return slice(0, self.n - (self.plane if self.upper else 0))


def halo_sum(v, slab, dist):
    """Adds the neighbours' partial values on the shared node planes of v (a
    1-D torch tensor of the slab's nodal values), in place: each rank sends
    its partial plane and adds the one it receives, so both sides end with
    the same sum (a + b on one side, b + a on the other; equal, since
    floating-point addition commutes)."""
    P = slab.plane
    reqs, recv = [], {}
    if slab.upper:
        recv["up"] = v.new_empty(P)
        reqs.append(dist.isend(v[-P:].contiguous(), slab.rank + 1))
        reqs.append(dist.irecv(recv["up"], slab.rank + 1))
    if slab.lower:
        recv["lo"] = v.new_empty(P)
        reqs.append(dist.isend(v[:P].contiguous(), slab.rank - 1))
        reqs.append(dist.irecv(recv["lo"], slab.rank - 1))
    for q in reqs:
        q.wait()
    if "up" in recv:
        v[-P:] += recv["up"]
    if "lo" in recv:
        v[:P] += recv["lo"]
    return v


def allreduce(vals, dist, like, op="sum"):
    """All-reduce of a few float64 scalars (one collective)."""
    import torch
    t = torch.tensor(vals, dtype=torch.float64, device=like.device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return t.tolist()


def pcg(slab, dist, apply_local, diag_local, free, b, tol=1e-6, max_iter=40000,
        shift_factor=0.0):
    """Distributed Jacobi-PCG on (K_ff + s I) u = b (b zero on fixed DOFs),
    s = shift_factor * max diag over free DOFs and M^-1 = 1 / (diag + s),
    stopping when ||r|| / ||b|| < tol (the recursive residual), as the
    single-domain solvers do.

    apply_local(x) -> partial K x on the slab's elements (torch tensor);
    diag_local -> partial diagonal; free -> 0/1 float mask of the slab's free
    DOFs (BC bits; nodes without stiffness are cleared here).  Returns
    (u, iterations, relative residual, shift)."""
    import torch
    own = slab.owned()
    d = halo_sum(diag_local.clone(), slab, dist)
    free = free * (d > 0).to(free.dtype)
    dmax = allreduce([float((d * free).max()) if free.numel() else 0.0], dist, d, "max")[0]
    s = shift_factor * dmax
    minv = torch.where(free > 0, 1.0 / (d + s), torch.zeros_like(d))

    def A(v):
        q = halo_sum(apply_local(v), slab, dist)
        return (q + s * v) * free

    x = torch.zeros_like(b)
    r = b * free
    z = minv * r
    p = z.clone()
    rz, bb = allreduce([float(r[own] @ z[own]), float(r[own] @ r[own])], dist, r)
    bnorm = bb ** 0.5
    if bnorm == 0.0:
        return x, 0, 0.0, s
    rel = 1.0
    it = 0
    for it in range(1, max_iter + 1):
        q = A(p)
        pq = allreduce([float(p[own] @ q[own])], dist, p)[0]
        if not (pq > 0.0):
            return x, -1, rel, s
        alpha = rz / pq
        x += alpha * p
        r -= alpha * q
        z = minv * r
        rzn, rr = allreduce([float(r[own] @ z[own]), float(r[own] @ r[own])], dist, r)
        rel = rr ** 0.5 / bnorm
        if rel < tol:
            break
        p = z + (rzn / rz) * p
        rz = rzn
    return x, it, rel, s


def gather(x, slab, dist):
    """The full nodal vector on every rank: the owned ranges of the ranks'
    slabs, concatenated in rank order (which is node order)."""
    import torch
    own = x[slab.owned()].contiguous()
    sizes = [None] * slab.world
    dist.all_gather_object(sizes, int(own.numel()))
    m = max(sizes)  # equal-size buffers (gloo needs them): pad, then trim
    pad = torch.zeros(m, dtype=x.dtype, device=x.device)
    pad[:own.numel()] = own
    bufs = [torch.zeros(m, dtype=x.dtype, device=x.device) for _ in sizes]
    dist.all_gather(bufs, pad)
    return torch.cat([b[:sz] for b, sz in zip(bufs, sizes)])


class DeviceSlabOperator:
    """The library's structured operator on this rank's slab (FP64 device
    tensors): K x through hx_apply_stiffness_noalloc on the slab's grid and
    element factors, on the current torch stream."""

    def __init__(self, slab, fac_slab, h=(1.0, 1.0, 1.0), nu=0.3):
        import torch
        from . import _lib
        self.L = _lib.load()
        self.slab = slab
        self.h, self.nu = h, nu
        self.fac = fac_slab.contiguous()
        self.y = torch.empty(slab.n, dtype=torch.float64, device=fac_slab.device)
        self.xkx = torch.zeros(1, dtype=torch.float64, device=fac_slab.device)

    def __call__(self, x):
        import ctypes
        import torch
        s = torch.cuda.current_stream(x.device)
        st = self.L.hx_apply_stiffness_noalloc(
            self.slab.nx, self.slab.ny, self.slab.nzl, *self.h, self.nu, x.data_ptr(),
            self.fac.data_ptr(), self.y.data_ptr(), self.xkx.data_ptr(),
            ctypes.c_void_p(s.cuda_stream))
        if st != 0:
            raise RuntimeError(f"hx_apply_stiffness_noalloc failed with status {st}")
        return self.y.clone()
