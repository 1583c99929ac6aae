"""The z-slab partitioned operator and CG (pmg.distributed) on CPU ranks over gloo.

Each rank computes its cells with the oracle (the CPU restatement, standing in for the GPU
kernels); the partition, the local renumbering, the ghost update and compress, the global
dot products and the distributed CG are the library's.  The partitioned vmult must equal the
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


class OracleBackend:
    """Local compute of one rank on the CPU oracle (test infrastructure)."""

    def __init__(self, part, p, O):
        from pmg.distributed import LocalNumbering
        ob = _obox(O, part.local_box())
        plain, cons, idx = O.dofs(ob, p)
        ijk, _ = O.dof_lattice(ob, p)
        self.numbering = nb = LocalNumbering(idx, cons, ijk, part)
        self.O, self.p = O, p
        self.G = O.geometry_G(ob, p)
        self.cons = np.zeros(nb.n, np.uint8)
        self.cons[nb.constrained] = 1

    def empty(self, n):
        return torch.empty(n, dtype=torch.float64)

    def zeros(self, n):
        return torch.zeros(n, dtype=torch.float64)

    def vmult(self, dst, src):
        dst.copy_(torch.from_numpy(self.O.vmult(self.p, self.numbering.dof_indices, self.G, self.cons, src.numpy())))

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
