"""Self-consistency of the oracle's cell operator: the BK3 collocation formulation against
the inverse-Jacobian formulation, a dense assembly (symmetry, SPD, diagonal), the coloured
parallel loop against the serial one, and the manufactured-solution convergence rate."""
import numpy as np
import pytest


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("deform", [0, 1])
def test_bk3_matches_invjac_formulation(oracle, p, deform):
    box = oracle.Box.make(refine=1, deform=deform)
    plain, cons, idx = oracle.dofs(box, p)
    G = oracle.geometry_G(box, p)
    iJ, jxw = oracle.invjac(box, p)
    src = np.random.default_rng(p).uniform(-1, 1, cons.shape[0])
    a = oracle.vmult(p, idx, G, cons, src)
    b = oracle.vmult_invjac(p, idx, iJ, jxw, cons, src)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    c = oracle.vmult(p, idx, G, cons, src, color=oracle.colors(box))
    assert np.abs(a - c).max() <= 1e-14 * np.abs(a).max()


@pytest.mark.parametrize("p", [1, 2, 4])
def test_dense_operator_symmetric_spd_and_diagonal(oracle, p):
    box = oracle.Box.make(coarse=(2, 1, 1), refine=1, deform=1, hi=(2, 1, 1))
    plain, cons, idx = oracle.dofs(box, p)
    G = oracle.geometry_G(box, p, coeff_kind=1)
    N = cons.shape[0]
    A = np.zeros((N, N))
    for j in range(N):
        e = np.zeros(N)
        e[j] = 1
        A[:, j] = oracle.vmult(p, idx, G, cons, e)
    np.testing.assert_allclose(A, A.T, atol=1e-13 * np.abs(A).max())
    assert np.linalg.eigvalsh(0.5 * (A + A.T)).min() > 0
    np.testing.assert_allclose(oracle.diagonal(p, idx, G, cons), np.diag(A), rtol=1e-13, atol=1e-15)


def test_numbering_first_visit(oracle):
    box = oracle.Box.make(coarse=(2, 1, 1), refine=1, hi=(2, 1, 1))
    for p in (1, 2, 3):
        plain, cons, idx = oracle.dofs(box, p)
        nm = p + 1
        N = (p * 4 + 1) * (p * 2 + 1) ** 2
        assert cons.shape[0] == N
        flat = plain.reshape(-1)
        # first-visit numbering: the first occurrence of every DoF number is in increasing order
        _, first = np.unique(flat, return_index=True)
        assert np.all(np.diff(first) > 0)
        assert set(np.unique(flat)) == set(range(N))
        # interior count
        assert int((cons == 0).sum()) == (p * 4 - 1) * (p * 2 - 1) ** 2
        assert np.all((idx == oracle.INVALID) == (cons[plain] == 1))


@pytest.mark.parametrize("p", [1, 2, 3])
def test_manufactured_solution_convergence(oracle, p):
    errs = []
    for r in (1, 2, 3):
        box = oracle.Box.make(refine=r)
        info, _ = oracle.solve_box(box, list(range(p, 0, -1)), cheb=3, rhs_kind=1, reduce=1e-12)
        errs.append(info.l2_error)
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert rates[-1] > p + 1 - 0.35, (errs, rates)


def test_plain_q2_h_multigrid_oracle(oracle):
    """The plain method (FE_Q(2), geometric multigrid at degree 2 on every level down to 2^3
    cells, Chebyshev(3), CG to 1e-10): a few iterations independent of the mesh size, and the
    L2 error falling like h^3 between 8^3 and 16^3 cells."""
    infos = []
    for refine in (2, 3):
        info, _ = oracle.solve_box(oracle.Box.make(coarse=(2, 2, 2), refine=refine), [2], cheb=3,
                                   rhs_kind=1, reduce=1e-10, h_degree=2)
        assert info.n_levels == refine + 1
        assert all(info.level_degree[l] == 2 for l in range(info.n_levels))
        infos.append(info)
    assert infos[1].n_dofs == 35937
    assert [i.iterations for i in infos] == [7, 7]
    assert 2.9 < np.log2(infos[0].l2_error / infos[1].l2_error) < 3.1
    with pytest.raises(ValueError):
        oracle.solve_box(oracle.Box.make(refine=1), [2, 1], h_degree=2)
