"""Operators, multigrid and CG sharded over GPUs: a z-slab partition of a box mesh, one rank
per GPU.

The reference distributes the cells over MPI ranks and, in every vmult, updates the ghost
DoFs of the source vector before the cell loop and adds the ghost contributions of the
destination back to their owners after it (LaplaceOperatorBK3::vmult,
include/operators/portable_laplace_operator_bk3.h:187-227, with the partitioner of deal.II's
MatrixFree); its transfers exchange the ghosts of the vector they read and compress the one
they write (include/multigrid/portable_geometric_transfer_core.h:23-157), and CG and the
Chebyshev eigenvalue estimate reduce their dot products over all ranks.  Here:

* `SlabPartition` gives rank r the coarse cells with z in [z_r, z_{r+1}) of the box and all
  their refinements: a box of its own (the interface faces are not Dirichlet faces), so every
  multigrid level and the geometry of the deformed map are partitioned the same way and the
  patch of an h-transfer never leaves a rank.
* `LocalNumbering` renumbers a rank's DoFs so that the interface planes are contiguous: the
  bottom plane (shared with rank r-1, owned here) first, the top plane (owned by rank r+1,
  ghosts here) last, each ordered by lattice (y, x) with its free DoFs before its Dirichlet
  ones.  Both neighbours list a plane in the same order, so the halo exchange moves
  contiguous vector slices, with no packing kernel, and the owned DoFs are the prefix
  [0, n_owned) over which the dot products run.
* `DistributedOperator` applies A with the ghost update (rank r+1 sends its bottom plane to
  rank r) and the compress (rank r sends the free entries of its top plane to r+1, which adds
  them to its bottom plane), point to point over torch.distributed (NCCL on GPUs, gloo on
  CPUs); the cells that read no ghost DoFs (all but the top layer, which `LocalNumbering`
  puts last in the cell order) are computed while the ghost update is in flight; `dot` is
  one FP64 all-reduce.
* `DistributedTransfer` uses the patch maps of each rank's cells with weights 1 / (patches
  holding the fine DoF over all ranks), `DistributedChebyshev` is deal.II's
  PreconditionChebyshev with global dot products in its eigenvalue estimate (start vector
  (g mod 11) - mean with g the DoF's global node-lattice index, independent of the
  partition), `DistributedMultigrid` the V-cycle of the single-GPU library over them, and
  `cg_solve` deal.II's SolverCG with ReductionControl, Jacobi- or V-cycle-preconditioned.

The local compute goes through a backend: `LibraryBackend` (this library's CUDA kernels, the
rank's operator built from its renumbered maps with pmg_operator_create_from_maps, transfers
with pmg_transfer_create_from_maps) on GPUs.  Every rank takes the same collective steps in
the same order."""
from __future__ import annotations

import numpy as np

from . import (F32, F64, GEOMETRY_FULL, TRANSFER_GEOMETRIC, TRANSFER_POLYNOMIAL, Box, LaplaceOperator, Mesh,
               Transfer, vector_axpy, vector_chebyshev_step, vector_copy, vector_dot, vector_pointwise_mult,
               vector_xpay)

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

    def global_lattice(self, degree, refine=None):
        """Node-lattice extents (x, y, z) of the whole box at this degree and refinement."""
        r = self.box.refine if refine is None else refine
        return tuple(degree * (c << r) + 1 for c in self.box.coarse)


class LocalNumbering:
    """The renumbering of one rank's DoFs (see the module docstring).

    dof_indices [C, nm^3] (sentinel on constrained DoFs), constrained [N] flags and lattice [N, 3]
    (node-lattice coordinates) describe the rank's box operator, cell_xyz [C, 3] its cells;
    `perm[old] = new`.  `plain` is the renumbered cell -> DoF map without the sentinel and
    `node` the local node lattice -> renumbered DoF."""

    def __init__(self, dof_indices, constrained, lattice, part: SlabPartition, cell_xyz=None, degree=None):
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
        # cells that read ghost DoFs (the top layer) last: the others are computed while the
        # ghost update is in flight
        cells = self.dof_indices if self.dof_indices.ndim == 2 else self.dof_indices.reshape(-1, (degree + 1) ** 3)
        touch = ((cells != INVALID) & (cells >= self.top_begin)).any(axis=1) if self.n_top else \
            np.zeros(cells.shape[0], bool)
        self.cell_order = np.concatenate([np.nonzero(~touch)[0], np.nonzero(touch)[0]]).astype(np.int64)
        self.n_inner_cells = int((~touch).sum())
        self.constrained = self.perm[np.nonzero(cons)[0]].astype(np.uint32)
        self.constrained_flags = np.zeros(n, bool)
        self.constrained_flags[self.constrained] = True
        self.lattice = np.empty_like(lat)
        self.lattice[self.perm] = lat
        if cell_xyz is not None:
            p, nm = degree, degree + 1
            extent = lat.max(axis=0) + 1 if n else np.zeros(3, np.int64)
            self.node = np.zeros((extent[2], extent[1], extent[0]), np.uint32)
            self.node[self.lattice[:, 2], self.lattice[:, 1], self.lattice[:, 0]] = np.arange(n, dtype=np.uint32)
            xyz = np.asarray(cell_xyz, dtype=np.int64)
            k, j, i = np.meshgrid(np.arange(nm), np.arange(nm), np.arange(nm), indexing="ij")
            self.cell_xyz = xyz
            self.plain = self.node[p * xyz[:, 2, None] + k.reshape(1, -1), p * xyz[:, 1, None] + j.reshape(1, -1),
                                   p * xyz[:, 0, None] + i.reshape(1, -1)]

    def global_index(self, part: SlabPartition, degree, refine=None):
        """Global lexicographic node-lattice index (x fastest) of every local DoF."""
        Lx, Ly, _ = part.global_lattice(degree, refine)
        zoff = part.z_offset(degree, refine)
        lat = self.lattice.astype(np.int64)
        return lat[:, 0] + Lx * (lat[:, 1] + Ly * (lat[:, 2] + zoff))


def transfer_maps(coarse: LocalNumbering, fine: LocalNumbering, degree_c, degree_f, h_transfer):
    """The patch maps of one rank's transfer in the renumbered numberings: one patch per cell
    (polynomial) or per coarse cell with the (2p+1)^3 fine nodes of its children (geometric)."""
    if not h_transfer:
        return TRANSFER_POLYNOMIAL, coarse.dof_indices, fine.plain
    p, nf = degree_c, 2 * degree_c + 1
    k, j, i = np.meshgrid(np.arange(nf), np.arange(nf), np.arange(nf), indexing="ij")
    xyz = coarse.cell_xyz
    fi = fine.node[2 * p * xyz[:, 2, None] + k.reshape(1, -1), 2 * p * xyz[:, 1, None] + j.reshape(1, -1),
                   2 * p * xyz[:, 0, None] + i.reshape(1, -1)]
    return TRANSFER_GEOMETRIC, coarse.dof_indices, fi


class LibraryBackend:
    """Local compute on this rank's GPU through libpmg_b200: the local operator from the
    renumbered maps, vectors as CUDA tensors, the library's vector kernels."""

    def __init__(self, part: SlabPartition, degree: int, dtype=F64, device=0, refine=None):
        import torch
        self.torch = torch
        self.device = device
        self.dtype = dtype
        self.degree = degree
        self.tdtype = torch.float64 if dtype == F64 else torch.float32
        mesh = Mesh(part.local_box(refine))
        box_op = LaplaceOperator(mesh, degree, dtype, GEOMETRY_FULL, device=device)
        self.numbering = LocalNumbering(box_op.dof_indices(), box_op.constrained(), box_op.dof_lattice(), part,
                                        mesh.cell_coordinates(), degree)
        geometry = box_op.geometry()
        del box_op
        nb = self.numbering
        n_cells = nb.cell_order.shape[0]
        # the operator holds the cells in the numbering's cell order (inner cells first)
        self.op = LaplaceOperator.from_maps(nb.n, nb.dof_indices.reshape(n_cells, -1)[nb.cell_order], nb.constrained,
                                            degree, dtype, G=geometry.reshape(n_cells, -1)[nb.cell_order],
                                            device=device)
        cpw = self.op.cells_per_group()
        self.n_cells = n_cells
        self.split = (nb.n_inner_cells // cpw) * cpw  # first cell of the boundary pass

    def empty(self, n):
        return self.torch.empty(n, dtype=self.tdtype, device=f"cuda:{self.device}")

    def zeros(self, n):
        return self.torch.zeros(n, dtype=self.tdtype, device=f"cuda:{self.device}")

    def from_host(self, a):
        return self.torch.as_tensor(np.asarray(a), dtype=self.tdtype).to(f"cuda:{self.device}")

    def to_host(self, v):
        return v.double().cpu().numpy()

    def vmult(self, dst, src):
        self.op.vmult(dst, src)

    def vmult_cells(self, dst, src, begin, end, init):
        self.op.vmult_cells(dst, src, begin, end, init)

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

    def zero(self, v):
        v.zero_()

    def reciprocal(self, v):
        """v = 1 / v in place (setup only)."""
        v.reciprocal_()

    def cheb_step(self, out, cur, prev, src, Ax, invd, f1, f2):
        vector_chebyshev_step(out, cur, prev, src, Ax, invd, f1, f2)

    def transfer(self, coarse_backend, kind, coarse_indices, fine_indices, weights):
        return Transfer.from_maps(coarse_backend.op, self.op, kind, coarse_indices, fine_indices, weights)


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
    def _post(self, sends, recvs):
        if not (self.dist.is_available() and self.dist.is_initialized()):
            return []
        ops = [self.dist.P2POp(self.dist.isend, t, peer) for t, peer in sends]
        ops += [self.dist.P2POp(self.dist.irecv, t, peer) for t, peer in recvs]
        return self.dist.batch_isend_irecv(ops) if ops else []

    def _exchange(self, sends, recvs):
        for req in self._post(sends, recvs):
            req.wait()

    def _ghost_ops(self, v):
        nb, r = self.nb, self.part.rank
        sends = [(v[:nb.n_bottom], r - 1)] if self.part.has_below else []
        recvs = [(v[nb.top_begin:], r + 1)] if self.part.has_above else []
        return sends, recvs

    def update_ghosts(self, v):
        """v's top plane (ghosts) := the owner's bottom plane."""
        self._exchange(*self._ghost_ops(v))

    def zero_ghosts(self, v):
        if self.nb.n_top:
            self.be.zero(v[self.nb.top_begin:])

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
        """dst = A src.  With a backend that applies cell ranges (`vmult_cells`, `split`), the
        cells that read no ghost DoFs are computed while the ghost update is in flight and the
        top layer after it (the reference's colour loop, bk3.h:187-227); the sends read only
        owned entries and the receives write only ghost entries, which the inner cells do not
        read."""
        split = getattr(self.be, "split", None)
        if split is None:
            self.update_ghosts(src)
            self.be.vmult(dst, src)
        else:
            reqs = self._post(*self._ghost_ops(src))
            self.be.vmult_cells(dst, src, 0, split, True)
            for req in reqs:
                req.wait()
            self.be.vmult_cells(dst, src, split, self.be.n_cells, False)
        self.compress(dst)

    def allreduce(self, values):
        import torch
        dev = "cpu" if getattr(self.be, "device", None) is None else f"cuda:{self.be.device}"
        t = torch.tensor(values, dtype=torch.float64, device=dev)
        if self.dist.is_available() and self.dist.is_initialized() and self.dist.get_world_size() > 1:
            self.dist.all_reduce(t)
        return [float(v) for v in t.cpu()]

    def dot(self, a, b):
        """Global a.b over the owned DoFs of every rank (one FP64 all-reduce)."""
        return self.allreduce([self.be.dot(a, b, self.n_owned)])[0]

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


class DistributedTransfer:
    """prolongate_and_add / restrict_and_add between two partitioned levels: the ghosts of the
    vector read are updated first, the entries written on ghost DoFs are compressed to their
    owners afterwards.  Weights 1 / (patches holding the fine DoF on all ranks), 0 on Dirichlet
    DoFs."""

    def __init__(self, coarse: DistributedOperator, fine: DistributedOperator, degree_c, degree_f, h_transfer):
        self.coarse, self.fine = coarse, fine
        kind, ci, fi = transfer_maps(coarse.nb, fine.nb, degree_c, degree_f, h_transfer)
        be = fine.be
        counts = be.from_host(np.bincount(np.asarray(fi, np.int64).reshape(-1), minlength=fine.n).astype(np.float64))
        fine.compress(counts)
        fine.update_ghosts(counts)
        mult = be.to_host(counts)
        w_dof = np.where(fine.nb.constrained_flags | (mult == 0), 0.0, 1.0 / np.maximum(mult, 1.0))
        self.local = fine.be.transfer(coarse.be, kind, ci, fi, w_dof[np.asarray(fi, np.int64)])

    def prolongate_and_add(self, dst_fine, src_coarse):
        self.coarse.update_ghosts(src_coarse)
        self.fine.zero_ghosts(dst_fine)
        self.local.prolongate_and_add(dst_fine, src_coarse)
        self.fine.compress(dst_fine)

    def restrict_and_add(self, dst_coarse, src_fine):
        self.fine.update_ghosts(src_fine)
        self.coarse.zero_ghosts(dst_coarse)
        self.local.restrict_and_add(dst_coarse, src_fine)
        self.coarse.compress(dst_coarse)


class DistributedChebyshev:
    """deal.II PreconditionChebyshev with the inverse diagonal, as the library's smoother
    (degree <= 0: chosen from smoothing_range), on a DistributedOperator."""

    def __init__(self, A: DistributedOperator, global_index, n_global, degree=5, smoothing_range=15.0,
                 eig_cg_n_iterations=10):
        self.A, self.be = A, A.be
        self.requested_degree, self.degree = degree, degree
        self.range, self.eig_its = smoothing_range, eig_cg_n_iterations
        self.gidx, self.n_global = np.asarray(global_index, np.int64), int(n_global)
        self.estimated = False
        n = A.n
        self.Ax, self.x1, self.x2, self.zero_v = self.be.empty(n), self.be.empty(n), self.be.empty(n), self.be.zeros(n)

    def estimate(self):
        """At most eig_cg_n_iterations CG steps (tolerance 1e-10) from x = 0 on
        v = (g mod 11) - mean with the Jacobi preconditioner; Lanczos matrix with deal.II's
        one-step lag; max scaled by 1.2."""
        A, be, n = self.A, self.be, self.A.n
        invd = A.inverse_diagonal()
        full, rem = divmod(self.n_global, 11)
        mean = (full * 55.0 + rem * (rem - 1) / 2) / self.n_global if self.n_global else 0.0
        r = be.from_host((self.gidx % 11).astype(np.float64) - mean)
        x, z, p, v = be.zeros(n), be.empty(n), be.empty(n), be.empty(n)
        res = np.sqrt(A.dot(r, r))
        diag, offd, it = [], [], 0
        if not res <= 1e-10 and self.eig_its > 0:
            be.mult(z, invd, r)
            rho = A.dot(r, z)
            rho_old, alpha, beta, eig_beta_alpha = rho, 0.0, 0.0, 0.0
            while True:
                it += 1
                if it > 1:
                    beta = rho / rho_old
                    be.xpay(p, beta, z)
                else:
                    be.copy(p, z)
                A.vmult(v, p)
                prev_alpha = alpha
                alpha = rho / A.dot(p, v)
                be.axpy(x, alpha, p)
                be.axpy(r, -alpha, v)
                res = np.sqrt(A.dot(r, r))
                rho_old = rho
                be.mult(z, invd, r)
                rho = A.dot(r, z)
                if it > 1:
                    diag.append(1.0 / prev_alpha + eig_beta_alpha)
                    eig_beta_alpha = beta / prev_alpha
                    offd.append(np.sqrt(beta) / prev_alpha)
                if it >= self.eig_its or res <= 1e-10:
                    break
        if diag:
            T = np.diag(diag) + np.diag(offd[:-1], 1) + np.diag(offd[:-1], -1)
            ev = np.linalg.eigvalsh(T)
            self.min_ev, self.max_ev = float(ev[0]), 1.2 * float(ev[-1])
        else:
            self.min_ev = self.max_ev = 1.0
        alpha_ev = self.max_ev / self.range if self.range > 1.0 else min(0.9 * self.max_ev, self.min_ev)
        if self.requested_degree <= 0:
            actual = self.max_ev / alpha_ev
            sigma = (1.0 - np.sqrt(1.0 / actual)) / (1.0 + np.sqrt(1.0 / actual))
            eps = self.range
            self.degree = 1 + int(np.log(1.0 / eps + np.sqrt(1.0 / eps / eps - 1.0)) / np.log(1.0 / sigma))
        self.delta = (self.max_ev - alpha_ev) * 0.5
        self.theta = (self.max_ev + alpha_ev) * 0.5
        self.cg_its = it
        self.estimated = True

    def apply(self, dst, src, from_zero):
        """vmult (from zero, degree-1 products) or step (from dst, degree products)."""
        if not self.estimated:
            self.estimate()
        A, be = self.A, self.be
        invd = A.inverse_diagonal()
        more = not (self.degree < 2 or abs(self.delta) < 1e-40)
        d = self.degree if more else 1
        if from_zero:
            be.cheb_step(dst, self.zero_v, None, src, self.zero_v, invd, 0.0, 1.0 / self.theta)
            cur, prev = dst, None
        else:
            A.vmult(self.Ax, dst)
            be.copy(self.x2, dst)
            be.cheb_step(self.x1, self.x2, None, src, self.Ax, invd, 0.0, 1.0 / self.theta)
            cur, prev = self.x1, self.x2
        if more:
            rhok, sigma = self.delta / self.theta, self.theta / self.delta
            spare = self.x1 if cur is dst else dst
            for _ in range(1, d):
                A.vmult(self.Ax, cur)
                rhokp = 1.0 / (2.0 * sigma - rhok)
                f1, f2 = rhokp * rhok, 2.0 * rhokp / self.delta
                rhok = rhokp
                out = prev if prev is not None else spare
                be.cheb_step(out, cur, prev, src, self.Ax, invd, f1, f2)
                prev, cur = cur, out
        if cur is not dst:
            be.copy(dst, cur)


class DistributedMultigrid:
    """The library's V-cycle (pre-smoothing from zero, residual, restriction, coarser cycle,
    prolongation, post-smoothing; the level-0 Chebyshev as the coarse solve) over partitioned
    levels; levels[0] is the coarsest."""

    def __init__(self, levels, transfers, smoothers):
        self.levels, self.transfers, self.smoothers = levels, transfers, smoothers
        self.sol = [lv.be.zeros(lv.n) for lv in levels]
        self.defect = [lv.be.zeros(lv.n) for lv in levels]
        self.t = [lv.be.zeros(lv.n) for lv in levels]

    def estimate(self):
        for s in self.smoothers:
            if not s.estimated:
                s.estimate()

    def _cycle(self, l):
        if l == 0:
            self.smoothers[0].apply(self.sol[0], self.defect[0], True)
            return
        lv, be = self.levels[l], self.levels[l].be
        self.smoothers[l].apply(self.sol[l], self.defect[l], True)
        lv.vmult(self.t[l], self.sol[l])
        be.xpay(self.t[l], -1.0, self.defect[l])  # t = defect - A sol
        self.levels[l - 1].be.zero(self.defect[l - 1])
        self.transfers[l].restrict_and_add(self.defect[l - 1], self.t[l])
        self._cycle(l - 1)
        self.transfers[l].prolongate_and_add(self.sol[l], self.sol[l - 1])
        self.smoothers[l].apply(self.sol[l], self.defect[l], False)

    def vmult(self, dst, src):
        """dst = V-cycle(src), converting precisions on entry and exit."""
        self.estimate()
        top = len(self.levels) - 1
        be = self.levels[top].be
        for l in range(top):
            self.levels[l].be.zero(self.defect[l])
        be.copy(self.defect[top], src)
        self._cycle(top)
        be.copy(dst, self.sol[top])


def build_hierarchy(part: SlabPartition, pseq, backend_factory, cheb_degree=5, smoothing_range=15.0,
                    eig_iterations=10, h_degree=1):
    """The multigrid hierarchy of pmg.Hierarchy on a partition: FE_Q(h_degree) on every
    refinement 0..box.refine, then the degrees of pseq (descending, ending in h_degree) on the
    finest mesh.  backend_factory(part, degree, refine) makes a level's local backend.
    Returns the DistributedMultigrid and the level operators."""
    R = part.box.refine
    specs = [(r, h_degree) for r in range(R + 1)] + [(R, p) for p in list(reversed(pseq))[1:]]
    levels, transfers, smoothers = [], [None], []
    for l, (r, p) in enumerate(specs):
        op = DistributedOperator(part, backend_factory(part, p, r))
        levels.append(op)
        gidx = op.nb.global_index(part, p, r)
        Lx, Ly, Lz = part.global_lattice(p, r)
        n_global = Lx * Ly * Lz
        if l == 0:
            smoothers.append(DistributedChebyshev(op, gidx, n_global, 0, 1e-3, n_global))
        else:
            smoothers.append(DistributedChebyshev(op, gidx, n_global, cheb_degree, smoothing_range, eig_iterations))
            rc, pc = specs[l - 1]
            transfers.append(DistributedTransfer(levels[l - 1], op, pc, p, h_transfer=rc != r))
    return DistributedMultigrid(levels, transfers, smoothers), levels


def cg_solve(A: DistributedOperator, x, b, reduce=1e-9, abs_tol=1e-16, max_iterations=100, precond=None):
    """CG on the distributed operator (deal.II SolverCG with ReductionControl(max_iterations,
    abs_tol, reduce), as the library's pmg_cg_solve), preconditioned by the Jacobi diagonal or
    a DistributedMultigrid: stops at the first iterate with ||r|| <= max(abs_tol, reduce
    ||r_0||).  x and b are this rank's local vectors (owned DoFs first, ghosts last); b's ghost
    entries are not read."""
    be, n = A.be, A.n
    invd = A.inverse_diagonal() if precond is None else None
    r, z, p, v = be.empty(n), be.empty(n), be.empty(n), be.empty(n)
    A.vmult(v, x)
    be.copy(r, b)
    be.axpy(r, -1.0, v)
    res = np.sqrt(A.dot(r, r))
    r0 = res
    tol = max(abs_tol, reduce * res)
    it, rho_old = 0, 0.0
    while res > tol and it < max_iterations:
        if precond is None:
            be.mult(z, invd, r)
        else:
            precond.vmult(z, r)
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
