"""Operators and CG sharded over GPUs: a z-slab partition of a box mesh, one rank per GPU.

The reference distributes the cells over MPI ranks and, in every vmult, updates the ghost
DoFs of the source vector before the cell loop and adds the ghost contributions of the
destination back to their owners after it (LaplaceOperatorBK3::vmult,
include/operators/portable_laplace_operator_bk3.h:187-227, with the partitioner of deal.II's
MatrixFree); CG reduces its dot products over all ranks.  Here:

* `SlabPartition` gives rank r the coarse cells with z in [z_r, z_{r+1}) of the box and all
  their refinements: a box of its own (the interface faces are not Dirichlet faces), so every
  multigrid level and the geometry of the deformed map are partitioned the same way.
* `LocalNumbering` renumbers a rank's DoFs so that the interface planes are contiguous: the
  bottom plane (shared with rank r-1, owned here) first, the top plane (owned by rank r+1,
  ghosts here) last, each ordered by lattice (y, x) with its free DoFs before its Dirichlet
  ones.  Both neighbours list a plane in the same order, so the halo exchange moves
  contiguous vector slices, with no packing kernel, and the owned DoFs are the prefix
  [0, n_owned) over which the dot products run.
* `DistributedOperator` applies A with the ghost update (rank r+1 sends its bottom plane to
  rank r) and the compress (rank r sends the free entries of its top plane to r+1, which adds
  them to its bottom plane), point to point over torch.distributed (NCCL on GPUs, gloo on
  CPUs); `dot` is one FP64 all-reduce.  `cg_solve` is the Jacobi-preconditioned CG of
  deal.II's SolverCG with ReductionControl on top of it.

The local compute goes through a backend: `LibraryBackend` (this library's CUDA kernels, the
local operator built from the renumbered maps with pmg_operator_create_from_maps) on GPUs.
Every rank takes the same collective steps in the same order."""
from __future__ import annotations

import numpy as np

from . import (F32, F64, GEOMETRY_FULL, Box, LaplaceOperator, Mesh, vector_axpy, vector_copy, vector_dot,
               vector_pointwise_mult, vector_xpay)

INVALID = 0xFFFFFFFF


class SlabPartition:
    """Rank `rank` of `world` owns the coarse z-cells [z_begin, z_end) of `box` (as even a split
    as the coarse cells allow; box.coarse[2] >= world) and every refinement of them."""

    def __init__(self, box: Box, world: int, rank: int):
        nz = box.coarse[2]
        if world < 1 or not 0 <= rank < world:
            raise ValueError("bad rank / world")
        if nz < world:
            raise ValueError(f"{nz} coarse cells along z cannot be split over {world} ranks")
        counts = [nz // world + (1 if r < nz % world else 0) for r in range(world)]
        self.box, self.world, self.rank = box, world, rank
        self.z_begin = sum(counts[:rank])
        self.z_end = self.z_begin + counts[rank]
        self.has_below, self.has_above = rank > 0, rank < world - 1

    def local_box(self, refine=None) -> Box:
        b = self.box
        hz = (b.hi[2] - b.lo[2]) / b.coarse[2]
        lo = (b.lo[0], b.lo[1], b.lo[2] + self.z_begin * hz)
        hi = (b.hi[0], b.hi[1], b.lo[2] + self.z_end * hz if self.has_above else b.hi[2])
        mask = b.dirichlet_mask
        if self.has_below:
            mask &= ~0x10
        if self.has_above:
            mask &= ~0x20
        return Box.make((b.coarse[0], b.coarse[1], self.z_end - self.z_begin), b.refine if refine is None else refine,
                        lo, hi, b.deform, b.amp, mask)

    def z_offset(self, degree, refine=None):
        """Global node-lattice z index of this rank's bottom plane."""
        r = self.box.refine if refine is None else refine
        return degree * (self.z_begin << r)


class LocalNumbering:
    """The caller-side renumbering of one rank's DoFs (see the module docstring).

    dof_indices [C, nm^3] (sentinel on constrained DoFs), constrained [N] flags and lattice [N, 3]
    describe the rank's box operator; `perm[old] = new`."""

    def __init__(self, dof_indices, constrained, lattice, part: SlabPartition):
        cons = np.asarray(constrained).astype(bool)
        lat = np.asarray(lattice)
        n = cons.shape[0]
        z = lat[:, 2]
        zmax = int(z.max()) if n else 0

        def plane(zval):
            ids = np.nonzero(z == zval)[0]
            key = np.lexsort((lat[ids, 0], lat[ids, 1], cons[ids]))  # free first, then (y, x)
            return ids[key]

        bottom = plane(0) if part.has_below else np.zeros(0, np.int64)
        top = plane(zmax) if part.has_above else np.zeros(0, np.int64)
        mark = np.zeros(n, bool)
        mark[bottom] = True
        mark[top] = True
        middle = np.nonzero(~mark)[0]
        order = np.concatenate([bottom, middle, top]).astype(np.int64)
        self.perm = np.empty(n, np.uint32)
        self.perm[order] = np.arange(n, dtype=np.uint32)
        self.n = n
        self.n_bottom, self.n_top = len(bottom), len(top)
        self.free_bottom = int((~cons[bottom]).sum())
        self.free_top = int((~cons[top]).sum())
        self.n_owned = n - self.n_top
        self.top_begin = n - self.n_top
        idx = np.asarray(dof_indices, dtype=np.uint32)
        self.dof_indices = np.where(idx == INVALID, np.uint32(INVALID),
                                    self.perm[np.minimum(idx, max(n - 1, 0))]).astype(np.uint32)
        self.constrained = self.perm[np.nonzero(cons)[0]].astype(np.uint32)
        self.lattice = np.empty_like(lat)
        self.lattice[self.perm] = lat


class LibraryBackend:
    """Local compute on this rank's GPU through libpmg_b200: the local operator from the
    renumbered maps, vectors as CUDA tensors, the library's vector kernels."""

    def __init__(self, part: SlabPartition, degree: int, dtype=F64, device=0):
        import torch
        self.torch = torch
        self.device = device
        self.dtype = dtype
        self.tdtype = torch.float64 if dtype == F64 else torch.float32
        box_op = LaplaceOperator(Mesh(part.local_box()), degree, dtype, GEOMETRY_FULL, device=device)
        self.numbering = LocalNumbering(box_op.dof_indices(), box_op.constrained(), box_op.dof_lattice(), part)
        geometry = box_op.geometry()
        del box_op
        nb = self.numbering
        self.op = LaplaceOperator.from_maps(nb.n, nb.dof_indices, nb.constrained, degree, dtype, G=geometry,
                                            device=device)

    def empty(self, n):
        return self.torch.empty(n, dtype=self.tdtype, device=f"cuda:{self.device}")

    def zeros(self, n):
        return self.torch.zeros(n, dtype=self.tdtype, device=f"cuda:{self.device}")

    def vmult(self, dst, src):
        self.op.vmult(dst, src)

    def inverse_diagonal(self):
        self.op.compute_diagonal()
        return self.op.get_matrix_diagonal_inverse()

    def dot(self, a, b, n):
        return vector_dot(a[:n], b[:n])

    def axpy(self, y, alpha, x):
        vector_axpy(y, x, alpha)

    def xpay(self, y, alpha, x):
        vector_xpay(y, x, alpha)

    def mult(self, z, d, r):
        vector_pointwise_mult(z, d, r)

    def copy(self, dst, src):
        vector_copy(dst, src)

    def reciprocal(self, v):
        """v = 1 / v in place (setup only)."""
        v.reciprocal_()


class DistributedOperator:
    """The global operator as seen by one rank: A restricted to this rank's cells, with the
    ghost update before and the compress after the local cell loop."""

    def __init__(self, part: SlabPartition, backend):
        import torch.distributed as dist
        self.dist = dist
        self.part, self.be = part, backend
        nb = backend.numbering
        self.nb = nb
        self.n, self.n_owned = nb.n, nb.n_owned
        self._inv_diag = None

    # -- halo exchange: every rank posts its sends and receives, then waits for all --------
    def _exchange(self, sends, recvs):
        ops = [self.dist.P2POp(self.dist.isend, t, peer) for t, peer in sends]
        ops += [self.dist.P2POp(self.dist.irecv, t, peer) for t, peer in recvs]
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()

    def update_ghosts(self, v):
        """v's top plane (ghosts) := the owner's bottom plane."""
        nb, r = self.nb, self.part.rank
        sends = [(v[:nb.n_bottom], r - 1)] if self.part.has_below else []
        recvs = [(v[nb.top_begin:], r + 1)] if self.part.has_above else []
        self._exchange(sends, recvs)

    def compress(self, v):
        """Adds the free entries of v's top plane (ghost contributions) to the owner's bottom
        plane; v's ghost entries are stale afterwards."""
        nb, r = self.nb, self.part.rank
        buf = self.be.empty(nb.free_bottom) if self.part.has_below else None
        sends = [(v[nb.top_begin:nb.top_begin + nb.free_top], r + 1)] if self.part.has_above else []
        recvs = [(buf, r - 1)] if self.part.has_below else []
        self._exchange(sends, recvs)
        if buf is not None and nb.free_bottom > 0:
            self.be.axpy(v[:nb.free_bottom], 1.0, buf)

    def vmult(self, dst, src):
        self.update_ghosts(src)
        self.be.vmult(dst, src)
        self.compress(dst)

    def dot(self, a, b):
        """Global a.b over the owned DoFs of every rank (one FP64 all-reduce)."""
        import torch
        local = self.be.dot(a, b, self.n_owned)
        t = torch.tensor([local], dtype=torch.float64, device=a.device)
        if self.dist.is_initialized() and self.dist.get_world_size() > 1:
            self.dist.all_reduce(t)
        return float(t.item())

    def inverse_diagonal(self):
        """1 / diag(A) on the owned DoFs (local diagonals summed across the interface), 1 on
        Dirichlet rows; ghost entries are made consistent too."""
        if self._inv_diag is None:
            d = self.be.inverse_diagonal()
            self.be.reciprocal(d)  # the local diagonal
            self.compress(d)
            self.update_ghosts(d)
            self.be.reciprocal(d)
            self._inv_diag = d
        return self._inv_diag


def cg_solve(A: DistributedOperator, x, b, reduce=1e-9, abs_tol=1e-16, max_iterations=100):
    """Jacobi-preconditioned CG on the distributed operator (deal.II SolverCG with
    ReductionControl(max_iterations, abs_tol, reduce), as the library's pmg_cg_solve): stops at
    the first iterate with ||r|| <= max(abs_tol, reduce ||r_0||).  x and b are this rank's
    local vectors (owned DoFs first, ghosts last); b's ghost entries are not read."""
    be, n = A.be, A.n
    invd = A.inverse_diagonal()
    r, z, p, v = be.empty(n), be.empty(n), be.empty(n), be.empty(n)
    A.vmult(v, x)
    be.copy(r, b)
    be.axpy(r, -1.0, v)
    res = np.sqrt(A.dot(r, r))
    r0 = res
    tol = max(abs_tol, reduce * res)
    it, rho_old = 0, 0.0
    while res > tol and it < max_iterations:
        be.mult(z, invd, r)
        rho = A.dot(r, z)
        if it == 0:
            be.copy(p, z)
        else:
            be.xpay(p, rho / rho_old, z)
        rho_old = rho
        it += 1
        A.vmult(v, p)
        pv = A.dot(p, v)
        if not pv > 0:
            raise RuntimeError("CG breakdown: p.Ap <= 0")
        alpha = rho / pv
        be.axpy(x, alpha, p)
        be.axpy(r, -alpha, v)
        res = np.sqrt(A.dot(r, r))
        if not np.isfinite(res):
            raise FloatingPointError("non-finite CG residual")
    return {"iterations": it, "converged": bool(res <= tol), "initial_residual": r0, "final_residual": res,
            "reduction_per_step": (res / r0) ** (1.0 / it) if it > 0 and r0 > 0 else 1.0}
