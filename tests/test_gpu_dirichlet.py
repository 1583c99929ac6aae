"""Inhomogeneous Dirichlet data by lifting (no counterpart in the reference, whose programs
impose homogeneous data, source/plain_solver/program.cc:125-131): the DoF support points
from pmg_operator_dof_coordinates against the node lattice restated here, the numbering of the
operator without Dirichlet DoFs against the constrained one, and the manufactured solution
u = exp(x) sin(pi y) cos(pi z) (nonzero on the boundary) recovered at the L2 rate p+1."""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu


def lattice_coords(oracle, box, p, plain, n):
    """Support points from the cell lattice and the GLL nodes, mapped by x' = x + a s(x)
    (s = sin(pi x) sin(pi y) sin(pi z), every component) on deformed boxes."""
    ob = oracle.Box.make(coarse=tuple(box.coarse), refine=box.refine, lo=tuple(box.lo), hi=tuple(box.hi),
                         deform=box.deform, amp=box.amp, dirichlet_mask=box.dirichlet_mask)
    cx, cy, cz = oracle.cell_coords(ob)
    xl, _ = oracle.gauss_lobatto(p + 1)
    ncell = [c << box.refine for c in box.coarse]
    h = [(box.hi[d] - box.lo[d]) / ncell[d] for d in range(3)]
    X = np.zeros((n, 3))
    nm = p + 1
    for c in range(ob.ncells()):
        for l in range(nm ** 3):
            i, j, k = l % nm, (l // nm) % nm, l // (nm * nm)
            x = np.array([box.lo[0] + (cx[c] + xl[i]) * h[0], box.lo[1] + (cy[c] + xl[j]) * h[1],
                          box.lo[2] + (cz[c] + xl[k]) * h[2]])
            if box.deform:
                x = x + box.amp * math.sin(math.pi * x[0]) * math.sin(math.pi * x[1]) * math.sin(math.pi * x[2])
            X[plain[c, l]] = x
    return X, ob


@pytest.mark.parametrize("p,deform", [(1, 0), (3, 0), (4, 1)])
def test_dof_coordinates_match_the_lattice(oracle, p, deform):
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0), deform=deform)
    op = pmg.LaplaceOperator(pmg.Mesh(box), p, pmg.F64)
    ob = oracle.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0), deform=deform)
    plain, cons, idx = oracle.dofs(ob, p)
    X, _ = lattice_coords(oracle, box, p, plain, cons.shape[0])
    got = op.dof_coordinates().cpu().numpy()
    assert np.abs(got - X).max() < 1e-13


def test_numbering_does_not_depend_on_the_dirichlet_dofs():
    b = pmg.Box.make(refine=2)
    free = pmg.Box.make(refine=2, dirichlet_mask=0)
    a = pmg.LaplaceOperator(pmg.Mesh(b), 3, pmg.F64)
    a0 = pmg.LaplaceOperator(pmg.Mesh(free), 3, pmg.F64)
    ia, i0 = a.dof_indices(), a0.dof_indices()
    assert a.m() == a0.m() and not (a0.constrained() != 0).any()
    keep = ia != pmg.INVALID
    np.testing.assert_array_equal(ia[keep], i0[keep])


def exact(xyz):
    return torch.exp(xyz[:, 0]) * torch.sin(math.pi * xyz[:, 1]) * torch.cos(math.pi * xyz[:, 2])


@pytest.mark.parametrize("p", [2, 3])
def test_lifting_recovers_the_manufactured_solution_at_rate_p_plus_1(p):
    errs = []
    for refine in (2, 3):
        h = pmg.Hierarchy(pmg.Box.make(refine=refine), sorted({p, 1}, reverse=True), mg_dtype=pmg.F32,
                          cheb_degree=4)
        b = h.fine64.assemble_rhs(2, p + 2)
        h.estimate()
        u, info = h.solve_dirichlet(b, exact, reduce=1e-12, max_iterations=200)
        assert info["converged"]
        errs.append(h.fine64.l2_error(u, 2))
        if refine == 3:
            # the boundary values are the data, and homogeneous data would be far off
            cons = torch.as_tensor(h.fine64.constrained().astype(bool), device="cuda")
            xyz = h.fine64.dof_coordinates()
            assert float((u[cons] - exact(xyz)[cons]).abs().max()) < 1e-14
            u_hom, _ = h.solve(b, reduce=1e-12, max_iterations=200)
            assert h.fine64.l2_error(u_hom, 2) > 100 * errs[-1]
    rate = math.log2(errs[0] / errs[1])
    assert rate > p + 0.5, (errs, rate)
