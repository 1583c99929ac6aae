"""Operators and transfers built from a caller's own discretisation (pmg_operator_create_from_maps,
pmg_transfer_create_from_maps), as a deal.II caller hands over its MatrixFree index map and
geometry (include/operators/portable_laplace_operator_bk3.h:360-437, :456-515) and its
transfer maps (include/base/portable_mg_transfer_base.h:32-36).

The caller's numbering here is the oracle's, with the DoF numbers of every level shuffled by
a random permutation and the cells of every level listed in a random order, so nothing
matches the library's own box numbering.  The library's results, mapped back through the
permutation, must equal the oracle's: vmult and the diagonal to 1e-12 (FP64) / 2e-5 (FP32),
a multigrid-preconditioned CG solve to the oracle's iteration count and solution."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu

INV = 0xFFFFFFFF
TOL = {pmg.F64: 1e-12, pmg.F32: 2e-5}


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def tdtype(dt):
    return torch.float64 if dt == pmg.F64 else torch.float32


def obox(oracle, b):
    return oracle.Box.make(coarse=tuple(b.coarse), refine=b.refine, lo=tuple(b.lo), hi=tuple(b.hi),
                           deform=b.deform, amp=b.amp, dirichlet_mask=b.dirichlet_mask)


class Shuffled:
    """One level of the oracle's discretisation in a caller's numbering: DoF d of the oracle
    is caller DoF perm[d]; caller cell c is oracle cell order[c]."""

    def __init__(self, oracle, box, p, seed):
        self.box, self.p = box, p
        self.plain, self.cons, self.idx = oracle.dofs(box, p)
        rng = np.random.default_rng(seed)
        self.n = self.cons.shape[0]
        self.perm = rng.permutation(self.n).astype(np.uint32)
        self.order = rng.permutation(self.idx.shape[0])
        self.oracle = oracle

    def map_dofs(self, a):
        a = np.asarray(a, dtype=np.uint32)
        return np.where(a == INV, np.uint32(INV), self.perm[np.minimum(a, self.n - 1)]).astype(np.uint32)

    def caller_indices(self):
        return self.map_dofs(self.idx[self.order])

    def caller_constrained(self):
        return self.perm[np.nonzero(self.cons)[0]]

    def to_caller(self, v):
        out = np.empty_like(v)
        out[self.perm] = v
        return out

    def from_caller(self, v):
        return v[self.perm]

    def operator(self, dtype, geometry="G"):
        O, nq3 = self.oracle, (self.p + 1) ** 3
        if geometry == "G":
            G = O.geometry_G(self.box, self.p)[self.order]
            return pmg.LaplaceOperator.from_maps(self.n, self.caller_indices(), self.caller_constrained(), self.p,
                                                 dtype, G=G)
        iJ, jxw = O.invjac(self.box, self.p)
        iJ = iJ.reshape(-1, nq3, 3, 3)[self.order]
        jxw = jxw.reshape(-1, nq3)[self.order]
        return pmg.LaplaceOperator.from_maps(self.n, self.caller_indices(), self.caller_constrained(), self.p,
                                             dtype, inv_jacobian=iJ, JxW=jxw)


def lattice_of(oracle, lvl):
    """Node lattice (z, y, x) -> oracle DoF of a level."""
    cx, cy, cz = oracle.cell_coords(lvl.box)
    p, nm = lvl.p, lvl.p + 1
    L = [p * (c << lvl.box.refine) + 1 for c in lvl.box.coarse]
    lat = np.zeros((L[2], L[1], L[0]), np.uint32)
    k, j, i = np.meshgrid(np.arange(nm), np.arange(nm), np.arange(nm), indexing="ij")
    for c in range(lvl.plain.shape[0]):
        lat[p * cz[c] + k, p * cy[c] + j, p * cx[c] + i] = lvl.plain[c].reshape(nm, nm, nm)
    return lat


def transfer_maps(oracle, coarse, fine, rng):
    """Caller patch maps between two shuffled levels, patches in a random order."""
    if coarse.box.refine == fine.box.refine:  # polynomial: one patch per cell
        ci, fi = coarse.idx, fine.plain
        kind = pmg.TRANSFER_POLYNOMIAL
    else:  # geometric: one patch per coarse cell, its 2p+1 fine nodes per direction
        p = coarse.p
        lat = lattice_of(oracle, fine)
        cx, cy, cz = oracle.cell_coords(coarse.box)
        nf = 2 * p + 1
        k, j, i = np.meshgrid(np.arange(nf), np.arange(nf), np.arange(nf), indexing="ij")
        fi = np.stack([lat[2 * p * cz[c] + k, 2 * p * cy[c] + j, 2 * p * cx[c] + i].reshape(-1)
                       for c in range(coarse.idx.shape[0])])
        ci = coarse.idx
        kind = pmg.TRANSFER_GEOMETRIC
    order = rng.permutation(ci.shape[0])
    return kind, coarse.map_dofs(ci[order]), fine.map_dofs(fi[order])


@pytest.mark.parametrize("p,dtype,geometry", [(4, pmg.F64, "G"), (4, pmg.F32, "G"), (2, pmg.F64, "G"),
                                              (3, pmg.F64, "INVJAC"), (3, pmg.F32, "INVJAC")])
def test_vmult_and_diagonal_in_caller_numbering(oracle, p, dtype, geometry):
    box = oracle.Box.make(refine=3, deform=1)
    lvl = Shuffled(oracle, box, p, seed=10 + p)
    op = lvl.operator(dtype, geometry)
    assert op.m() == lvl.n and op.n_cells() == lvl.idx.shape[0]
    np.testing.assert_array_equal(op.dof_indices(), lvl.caller_indices())
    src = np.random.default_rng(1234).uniform(-1, 1, lvl.n)
    G = oracle.geometry_G(box, p)
    want = oracle.vmult(p, lvl.idx, G, lvl.cons, src)
    d = op.initialize_dof_vector()
    op.vmult(d, torch.tensor(lvl.to_caller(src), dtype=tdtype(dtype), device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(lvl.from_caller(d.double().cpu().numpy()), want) < TOL[dtype]
    op.compute_diagonal()
    inv = op.get_matrix_diagonal_inverse()
    torch.cuda.synchronize()
    diag = oracle.diagonal(p, lvl.idx, G, lvl.cons)
    assert rel_err(1.0 / lvl.from_caller(inv.double().cpu().numpy()), diag) < 10 * TOL[dtype]


@pytest.mark.parametrize("mg_dtype", [pmg.F64, pmg.F32])
def test_multigrid_cg_in_caller_numbering_matches_oracle(oracle, mg_dtype):
    """ph-multigrid (Q1 h-levels on 1^3 .. 8^3 cells of the deformed cube, then Q2, Q4) with
    every level, transfer and the CG matrix built from shuffled caller maps."""
    box = oracle.Box.make(refine=3, deform=1)
    info_o, x_o = oracle.solve_box(box, [4, 2, 1], cheb=5, want_x=True)
    specs = [(r, 1) for r in range(4)] + [(3, 2), (3, 4)]
    levels = [Shuffled(oracle, oracle.Box.make(refine=r, deform=1), p, seed=100 + 7 * i)
              for i, (r, p) in enumerate(specs)]
    ops = [lv.operator(mg_dtype) for lv in levels]
    rng = np.random.default_rng(5)
    transfers = [None]
    for l in range(1, len(levels)):
        kind, ci, fi = transfer_maps(oracle, levels[l - 1], levels[l], rng)
        transfers.append(pmg.Transfer.from_maps(ops[l - 1], ops[l], kind, ci, fi))
    smoothers = [pmg.Chebyshev(ops[0], 0, 1e-3, ops[0].m())]
    smoothers += [pmg.Chebyshev(op, 5, 15.0, 10) for op in ops[1:]]
    mg = pmg.VCycleMultigrid(ops, transfers, smoothers)
    fine = levels[-1]
    A = fine.operator(pmg.F64)
    b = oracle.rhs(box, 4, 5, 0, fine.plain, fine.cons)
    x = A.initialize_dof_vector()
    info = pmg.solve_cg(A, x, torch.tensor(fine.to_caller(b), device="cuda"), mg)
    torch.cuda.synchronize()
    # the Chebyshev eigenvalue estimates start from (i mod 11) in the caller's numbering, so
    # the smoothers differ slightly from the oracle's: iterations within one, same solution
    assert info["converged"]
    assert abs(info["iterations"] - info_o.iterations) <= 1
    assert rel_err(fine.from_caller(x.cpu().numpy()), x_o) < 1e-8


def test_transfer_with_explicit_weights_equals_default(oracle):
    coarse = Shuffled(oracle, oracle.Box.make(refine=2), 2, seed=1)
    fine = Shuffled(oracle, oracle.Box.make(refine=2), 4, seed=2)
    oc, of = coarse.operator(pmg.F64), fine.operator(pmg.F64)
    kind, ci, fi = transfer_maps(oracle, coarse, fine, np.random.default_rng(0))
    mult = np.bincount(fi.reshape(-1), minlength=fine.n).astype(np.float64)
    cons = np.zeros(fine.n, bool)
    cons[fine.caller_constrained()] = True
    w = np.where(cons[fi], 0.0, 1.0 / mult[fi])
    t0 = pmg.Transfer.from_maps(oc, of, kind, ci, fi)
    t1 = pmg.Transfer.from_maps(oc, of, kind, ci, fi, weights=w)
    xc = torch.tensor(np.random.default_rng(3).uniform(-1, 1, coarse.n), device="cuda")
    y0, y1 = of.initialize_dof_vector(), of.initialize_dof_vector()
    t0.prolongate_and_add(y0, xc)
    t1.prolongate_and_add(y1, xc)
    torch.cuda.synchronize()
    assert rel_err(y1.cpu().numpy(), y0.cpu().numpy()) < 1e-15
    ref = oracle.transfer_apply(oracle.Box.make(refine=2), 2, 4, 0, coarse.from_caller(xc.cpu().numpy()),
                                np.zeros(fine.n))
    assert rel_err(fine.from_caller(y0.cpu().numpy()), ref) < 1e-13


def test_caller_maps_errors(oracle):
    lvl = Shuffled(oracle, oracle.Box.make(refine=1), 2, seed=3)
    bad = lvl.caller_indices().copy()
    bad[0, 0] = lvl.n  # out of range
    G = oracle.geometry_G(lvl.box, 2)[lvl.order]
    with pytest.raises(pmg.PmgError) as e:
        pmg.LaplaceOperator.from_maps(lvl.n, bad, lvl.caller_constrained(), 2, pmg.F64, G=G)
    assert e.value.status == -6
    op = lvl.operator(pmg.F64)
    with pytest.raises(pmg.PmgError) as e:  # no box mesh behind a caller-described operator
        op.assemble_rhs(0)
    assert e.value.status == -7
    with pytest.raises(pmg.PmgError) as e:  # box transfers need box operators
        pmg.Transfer(op, op)
    assert e.value.status == -1


def test_distributed_operator_on_one_gpu_equals_the_box_operator(oracle):
    """pmg.distributed with its CUDA backend at world size 1 (the renumbered caller-map
    operator, no neighbours): vmult and the Jacobi CG equal the box operator's."""
    import torch.distributed as dist
    from pmg.distributed import DistributedOperator, LibraryBackend, SlabPartition, cg_solve
    box = pmg.Box.make(coarse=(2, 2, 2), refine=2, deform=1)
    part = SlabPartition(box, 1, 0)
    be = LibraryBackend(part, 3, pmg.F64)
    A = DistributedOperator(part, be)
    assert not dist.is_initialized()
    ref = pmg.LaplaceOperator(pmg.Mesh(box), 3, pmg.F64, pmg.GEOMETRY_FULL)
    lat = ref.dof_lattice()
    ijk, _ = oracle.dof_lattice(obox(oracle, box), 3)
    np.testing.assert_array_equal(lat, ijk)
    # box DoF of every renumbered DoF
    perm = be.numbering.perm
    src = np.random.default_rng(9).uniform(-1, 1, ref.m())
    y_ref = ref.initialize_dof_vector()
    ref.vmult(y_ref, torch.tensor(src, device="cuda"))
    y = be.zeros(A.n)
    xs = np.empty_like(src)
    xs[perm] = src
    A.vmult(y, torch.tensor(xs, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(y.cpu().numpy()[perm], y_ref.cpu().numpy()) < 1e-12
    b = ref.assemble_rhs(1, 5)
    bs = torch.empty_like(b)
    bs[torch.as_tensor(perm.astype(np.int64), device="cuda")] = b
    x = be.zeros(A.n)
    info = cg_solve(A, x, bs, reduce=1e-10, max_iterations=1000)
    x_ref = ref.initialize_dof_vector()
    info_ref = pmg.solve_cg(ref, x_ref, b, None, reduce=1e-10, max_iterations=1000)
    assert info["converged"] and info["iterations"] == info_ref["iterations"]
    assert rel_err(x.cpu().numpy()[perm], x_ref.cpu().numpy()) < 1e-10
