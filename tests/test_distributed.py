"""The z-slab partitioned operator and CG (pmg.distributed) on CPU ranks over gloo.

Each rank computes its cells with the oracle (the CPU restatement, standing in for the GPU
kernels); the partition, the local renumbering, the ghost update and compress (with the inner
cells computed while the ghost update is in flight), the global dot products and the
distributed CG are the library's.  The partitioned vmult must equal the
single-domain oracle vmult to 1e-13, every global DoF must be owned by exactly one rank, and
the distributed Jacobi-CG must take the single-domain Jacobi-CG's iterations and give its
solution to 1e-10."""
import os
import socket
import sys
from datetime import timedelta

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
torch = pytest.importorskip("torch")

CASES = {
    # name: (coarse cells per direction, refine, degree, world)
    "q2_two_ranks": (2, 2, 2, 2),
    "q3_three_ranks": (3, 1, 3, 3),
}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _global_box(pmg, c, r):
    return pmg.Box.make(coarse=(c, c, c), refine=r, deform=1, amp=0.1)


def _obox(O, b):
    return O.Box.make(coarse=tuple(b.coarse), refine=b.refine, lo=tuple(b.lo), hi=tuple(b.hi), deform=b.deform,
                      amp=b.amp, dirichlet_mask=b.dirichlet_mask)


class NumpyTransfer:
    """A patch transfer with explicit weights in numpy (test infrastructure)."""

    def __init__(self, M, ci, fi, w):
        self.M = M  # [nc][nf]
        nc, nf = M.shape
        self.ci = np.asarray(ci, np.int64).reshape(-1, nc ** 3)
        self.fi = np.asarray(fi, np.int64).reshape(-1, nf ** 3)
        self.w = np.asarray(w, np.float64).reshape(self.fi.shape)
        self.valid = self.ci != 0xFFFFFFFF

    def prolongate_and_add(self, dst, src):
        nc, nf = self.M.shape
        s = src.numpy()
        c = np.where(self.valid, s[np.where(self.valid, self.ci, 0)], 0.0).reshape(-1, nc, nc, nc)
        f = np.einsum("pkji,ia,jb,kc->pcba", c, self.M, self.M, self.M).reshape(-1, nf ** 3)
        d = dst.numpy()
        np.add.at(d, self.fi.reshape(-1), (self.w * f).reshape(-1))

    def restrict_and_add(self, dst, src):
        nc, nf = self.M.shape
        f = (self.w * src.numpy()[self.fi]).reshape(-1, nf, nf, nf)
        c = np.einsum("pcba,ia,jb,kc->pkji", f, self.M, self.M, self.M).reshape(-1, nc ** 3)
        d = dst.numpy()
        np.add.at(d, self.ci[self.valid], c[self.valid])


class OracleBackend:
    """Local compute of one rank on the CPU oracle (test infrastructure)."""

    device = None

    def __init__(self, part, p, O, refine=None):
        from pmg.distributed import LocalNumbering
        ob = _obox(O, part.local_box(refine))
        plain, cons, idx = O.dofs(ob, p)
        ijk, _ = O.dof_lattice(ob, p)
        cx, cy, cz = O.cell_coords(ob)
        self.numbering = nb = LocalNumbering(idx, cons, ijk, part, np.stack([cx, cy, cz], axis=1), p)
        self.O, self.p = O, p
        self.G = O.geometry_G(ob, p)
        self.cons = np.zeros(nb.n, np.uint8)
        self.cons[nb.constrained] = 1
        # the cell order of the library backend (inner cells first) and its split at a multiple
        # of the cells per warp group, so that DistributedOperator.vmult takes the overlapped
        # path (inner cells during the ghost update, the top layer after it)
        self.n_cells = nb.cell_order.shape[0]
        cpw = 32 // (p + 1)
        self.split = (nb.n_inner_cells // cpw) * cpw
        self.calls = []

    def from_host(self, a):
        return torch.tensor(np.asarray(a, np.float64))

    def to_host(self, v):
        return v.numpy().copy()

    def zero(self, v):
        v.zero_()

    def cheb_step(self, out, cur, prev, src, Ax, invd, f1, f2):
        pv = torch.zeros_like(cur) if prev is None else prev
        out.copy_(cur + f1 * (cur - pv) + f2 * invd * (src - Ax))

    def transfer(self, coarse_backend, kind, ci, fi, weights):
        import pmg
        pc, pf = coarse_backend.p, self.p
        M = self.O.projection_matrix(pc, pf) if kind == pmg.TRANSFER_POLYNOMIAL else self.O.h_prolongation_matrix(pc)
        return NumpyTransfer(M, ci, fi, weights)

    def empty(self, n):
        return torch.empty(n, dtype=torch.float64)

    def zeros(self, n):
        return torch.zeros(n, dtype=torch.float64)

    def vmult(self, dst, src):
        dst.copy_(torch.from_numpy(self.O.vmult(self.p, self.numbering.dof_indices, self.G, self.cons, src.numpy())))

    def vmult_cells(self, dst, src, begin, end, init):
        """dst += A_K src over the cells [begin, end) of the cell order (init: dst = that with
        the identity rows), as pmg_operator_vmult_cells."""
        self.calls.append((begin, end, init))
        cells = self.numbering.cell_order[begin:end]
        idx = self.numbering.dof_indices.reshape(self.n_cells, -1)[cells]
        G = self.G.reshape(self.n_cells, -1)[cells]
        s = src.numpy()
        y = self.O.vmult(self.p, idx, G, self.cons, s)
        if init:
            dst.copy_(torch.from_numpy(y))
        else:
            y[self.cons == 1] -= s[self.cons == 1]  # the identity rows only once
            dst.add_(torch.from_numpy(y))

    def inverse_diagonal(self):
        d = self.O.diagonal(self.p, self.numbering.dof_indices, self.G, self.cons)
        inv = np.where(self.cons == 1, 1.0, 1.0 / np.where(d == 0, 1.0, d))
        return torch.from_numpy(inv)

    def dot(self, a, b, n):
        return float(a[:n].dot(b[:n]))

    def axpy(self, y, alpha, x):
        y.add_(x, alpha=alpha)

    def xpay(self, y, alpha, x):
        y.mul_(alpha).add_(x)

    def mult(self, z, d, r):
        torch.mul(d, r, out=z)

    def copy(self, dst, src):
        dst.copy_(src)

    def reciprocal(self, v):
        v.reciprocal_()


def _worker(rank, world, port, q, case):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    for p in (ROOT, os.path.join(ROOT, "portable-multigrid_b200")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import pmg
        from pmg.distributed import DistributedOperator, SlabPartition, cg_solve
        from oracle import oracle as O
        c, r, p, _ = CASES[case]
        gbox = _global_box(pmg, c, r)
        part = SlabPartition(gbox, world, rank)
        be = OracleBackend(part, p, O)
        A = DistributedOperator(part, be)
        nb = be.numbering
        _, glat = O.dof_lattice(_obox(O, gbox), p)
        zoff = part.z_offset(p)
        gid = glat[nb.lattice[:, 2] + zoff, nb.lattice[:, 1], nb.lattice[:, 0]].astype(np.int64)
        n_global = int(glat.max()) + 1
        src = np.random.default_rng(1234).uniform(-1, 1, n_global)
        dst = be.empty(nb.n)
        A.vmult(dst, torch.from_numpy(src[gid].copy()))
        plain_g, cons_g, _ = O.dofs(_obox(O, gbox), p)
        b_g = O.rhs(_obox(O, gbox), p, p + 1, 0, plain_g, cons_g)
        x = be.zeros(nb.n)
        info = cg_solve(A, x, torch.from_numpy(b_g[gid].copy()), reduce=1e-10, max_iterations=500)
        # the overlapped path: an inner pass with init, then the boundary pass; with ghosts the
        # top layer is a proper part of the cells
        assert be.calls[:2] == [(0, be.split, True), (be.split, be.n_cells, False)]
        if part.has_above:
            assert 0 < be.split < be.n_cells
            top = set(be.numbering.cell_order[nb.n_inner_cells:].tolist())
            di = nb.dof_indices.reshape(be.n_cells, -1)
            reads_ghost = ((di != 0xFFFFFFFF) & (di >= nb.top_begin)).any(axis=1)
            assert top == set(np.nonzero(reads_ghost)[0].tolist())
        q.put((rank, gid[:nb.n_owned], dst[:nb.n_owned].numpy(), x[:nb.n_owned].numpy(), info,
               (nb.n_bottom, nb.n_top, nb.free_bottom, nb.free_top)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _single_domain_jacobi_cg(O, box, p, b, reduce):
    plain, cons, idx = O.dofs(box, p)
    G = O.geometry_G(box, p)
    d = O.diagonal(p, idx, G, cons)
    invd = np.where(cons == 1, 1.0, 1.0 / d)
    x = np.zeros_like(b)
    r = b - O.vmult(p, idx, G, cons, x)
    res = np.sqrt(r @ r)
    tol = max(1e-16, reduce * res)
    it, rho_old, pv = 0, 0.0, None
    while res > tol and it < 500:
        z = invd * r
        rho = r @ z
        pv = z.copy() if it == 0 else z + (rho / rho_old) * pv
        rho_old = rho
        it += 1
        v = O.vmult(p, idx, G, cons, pv)
        alpha = rho / (pv @ v)
        x += alpha * pv
        r -= alpha * v
        res = np.sqrt(r @ r)
    return x, it


@pytest.mark.parametrize("case", sorted(CASES))
def test_slab_partitioned_vmult_and_cg_equal_single_domain(oracle, case):
    import torch.multiprocessing as mp
    import pmg
    c, r, p, world = CASES[case]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(k, world, port, q, case)) for k in range(world)]
    for pr in procs:
        pr.start()
    got = sorted([q.get(timeout=300) for _ in procs], key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    gbox = _obox(oracle, _global_box(pmg, c, r))
    plain, cons, idx = oracle.dofs(gbox, p)
    n = cons.shape[0]
    # every global DoF owned by exactly one rank
    owned = np.concatenate([g[1] for g in got])
    assert np.array_equal(np.sort(owned), np.arange(n))
    # the interface planes match between neighbours
    for k in range(world - 1):
        assert got[k][5][1] == got[k + 1][5][0] and got[k][5][3] == got[k + 1][5][2]
    src = np.random.default_rng(1234).uniform(-1, 1, n)
    want = oracle.vmult(p, idx, oracle.geometry_G(gbox, p), cons, src)
    y = np.zeros(n)
    for g in got:
        y[g[1]] = g[2]
    assert np.abs(y - want).max() <= 1e-13 * np.abs(want).max()
    b = oracle.rhs(gbox, p, p + 1, 0, plain, cons)
    x_ref, its_ref = _single_domain_jacobi_cg(oracle, gbox, p, b, 1e-10)
    x = np.zeros(n)
    for g in got:
        x[g[1]] = g[3]
        assert g[4]["converged"]
        assert g[4]["iterations"] == its_ref
    assert np.abs(x - x_ref).max() <= 1e-10 * np.abs(x_ref).max()


def test_partition_boxes_tile_the_global_box():
    sys.path.insert(0, os.path.join(ROOT, "portable-multigrid_b200"))
    import pmg
    from pmg.distributed import SlabPartition
    box = pmg.Box.make(coarse=(2, 2, 5), refine=1, hi=(1.0, 1.0, 2.5), dirichlet_mask=0x3F)
    parts = [SlabPartition(box, 3, r) for r in range(3)]
    assert [(pt.z_begin, pt.z_end) for pt in parts] == [(0, 2), (2, 4), (4, 5)]
    boxes = [pt.local_box() for pt in parts]
    assert boxes[0].lo[2] == 0.0 and boxes[-1].hi[2] == 2.5
    for a, b in zip(boxes, boxes[1:]):
        assert a.hi[2] == pytest.approx(b.lo[2])
    assert [bx.dirichlet_mask for bx in boxes] == [0x1F, 0x0F, 0x2F]
    assert parts[1].z_offset(3) == 3 * (2 << 1)
    with pytest.raises(ValueError):
        SlabPartition(pmg.Box.make(coarse=(1, 1, 2)), 3, 0)


MG_CASES = {
    # name: (coarse cells per direction, refine, pseq, Chebyshev degree)
    "q2_phmg": (2, 2, [2, 1], 3),
    "q3_phmg": (3, 1, [3, 1], 4),
}


def _mg_worker(rank, world, port, q, case):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    for p in (ROOT, os.path.join(ROOT, "portable-multigrid_b200")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        import pmg
        from pmg.distributed import DistributedOperator, SlabPartition, build_hierarchy, cg_solve
        from oracle import oracle as O
        c, r, pseq, cheb = MG_CASES[case]
        gbox = _global_box(pmg, c, r)
        part = SlabPartition(gbox, world, rank)
        mg, levels = build_hierarchy(part, pseq, lambda pt, p, rr: OracleBackend(pt, p, O, rr), cheb_degree=cheb)
        p = pseq[0]
        A = DistributedOperator(part, OracleBackend(part, p, O))
        nb = A.nb
        _, glat = O.dof_lattice(_obox(O, gbox), p)
        gid = glat[nb.lattice[:, 2] + part.z_offset(p), nb.lattice[:, 1], nb.lattice[:, 0]].astype(np.int64)
        plain_g, cons_g, _ = O.dofs(_obox(O, gbox), p)
        b_g = O.rhs(_obox(O, gbox), p, p + 1, 0, plain_g, cons_g)
        x = torch.zeros(nb.n, dtype=torch.float64)
        info = cg_solve(A, x, torch.from_numpy(b_g[gid].copy()), reduce=1e-10, max_iterations=100, precond=mg)
        evs = [(s.min_ev, s.max_ev, s.degree) for s in mg.smoothers]
        q.put((rank, gid[:nb.n_owned], x[:nb.n_owned].numpy(), info, evs))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run_mg(case, world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mg_worker, args=(k, world, port, q, case)) for k in range(world)]
    for pr in procs:
        pr.start()
    got = sorted([q.get(timeout=600) for _ in procs], key=lambda t: t[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    return got


@pytest.mark.parametrize("case,world", [("q2_phmg", 2), ("q3_phmg", 3)])
def test_slab_partitioned_vcycle_cg_equals_one_rank(oracle, case, world):
    """The V-cycle-preconditioned CG on 2 / 3 ranks takes the iterations of the same solver on
    one rank and gives its solution to 1e-10; the smoothers' eigenvalue estimates agree to
    1e-10; the one-rank solve is within one iteration of the oracle's single-domain solver."""
    import pmg
    c, r, pseq, cheb = MG_CASES[case]
    one = _run_mg(case, 1)
    many = _run_mg(case, world)
    gbox = _obox(oracle, _global_box(pmg, c, r))
    n = oracle.dofs(gbox, pseq[0])[1].shape[0]
    xs = []
    for got in (one, many):
        x = np.zeros(n)
        owned = np.concatenate([g[1] for g in got])
        assert np.array_equal(np.sort(owned), np.arange(n))
        for g in got:
            x[g[1]] = g[2]
            assert g[3]["converged"]
        xs.append(x)
    its1 = one[0][3]["iterations"]
    assert all(g[3]["iterations"] == its1 for g in many)
    assert np.abs(xs[1] - xs[0]).max() <= 1e-10 * np.abs(xs[0]).max()
    for (mn1, mx1, d1), (mn2, mx2, d2) in zip(one[0][4], many[0][4]):
        assert d1 == d2 and abs(mx2 / mx1 - 1) < 1e-10 and abs(mn2 / mn1 - 1) < 1e-8
    info_o, x_o = oracle.solve_box(gbox, pseq, cheb=cheb, reduce=1e-10, want_x=True)
    assert abs(its1 - info_o.iterations) <= 1
    assert np.abs(xs[0] - x_o).max() <= 1e-8 * np.abs(x_o).max()
