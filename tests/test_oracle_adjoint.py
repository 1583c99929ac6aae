"""Pins of the oracle's adjoint-path restatement (mass matrix, per-point form, coefficient
interpolation, adjoint gradient).  None of it is in the reference, so the pins are
mathematical: exact integrals of polynomials, the identity sum_q form(u, v) = u^T A v with the
oracle's Laplace vmult, exactness of the interpolation on polynomial log-fields, and central
finite differences of J(m) = 1/2 ||u(m) - u_d||^2 against the adjoint gradient."""
import numpy as np
import pytest

from pmg.adjoint import fourier_field


def node_coords(oracle, box, p, plain, N):
    """Coordinates of every DoF (undeformed box): cell lattice + GLL nodes."""
    cx, cy, cz = oracle.cell_coords(box)
    xl, _ = oracle.gauss_lobatto(p + 1)
    n = [c << box.refine for c in box.coarse]
    h = [(box.hi[d] - box.lo[d]) / n[d] for d in range(3)]
    X = np.zeros((N, 3))
    nm = p + 1
    for c in range(box.ncells()):
        for l in range(nm ** 3):
            i, j, k = l % nm, (l // nm) % nm, l // (nm * nm)
            X[plain[c, l]] = [box.lo[0] + (cx[c] + xl[i]) * h[0], box.lo[1] + (cy[c] + xl[j]) * h[1],
                              box.lo[2] + (cz[c] + xl[k]) * h[2]]
    return X


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_mass_integrates_polynomials_exactly(oracle, p):
    box = oracle.Box.make(coarse=(2, 1, 1), refine=1, lo=(0.0, -1.0, 0.0), hi=(2.0, 1.0, 0.5),
                          dirichlet_mask=0)
    plain, cons, idx = oracle.dofs(box, p)
    _, jxw = oracle.quadrature(box, p)
    X = node_coords(oracle, box, p, plain, cons.shape[0])
    # u = x^a y^b z^c with a, b, c <= p is represented exactly; int u^2 exactly integrated
    a, b, c = min(p, 2), min(p, 1), p
    u = X[:, 0] ** a * X[:, 1] ** b * X[:, 2] ** c
    exact = (2.0 ** (2 * a + 1) / (2 * a + 1)) * ((1.0 - (-1.0) ** (2 * b + 1)) / (2 * b + 1)) \
        * (0.5 ** (2 * c + 1) / (2 * c + 1))
    got = u @ oracle.mass_vmult(p, idx, jxw, cons, u)
    assert abs(got - exact) <= 1e-12 * abs(exact)
    # diagonal against unit vectors
    d = oracle.mass_diagonal(p, idx, jxw, cons)
    rng = np.random.default_rng(p)
    for i in rng.choice(cons.shape[0], 5, replace=False):
        e = np.zeros(cons.shape[0])
        e[i] = 1.0
        assert abs(oracle.mass_vmult(p, idx, jxw, cons, e)[i] - d[i]) <= 1e-13 * abs(d[i])


@pytest.mark.parametrize("p,deform", [(2, 0), (3, 1), (4, 0)])
def test_qp_form_sums_to_the_bilinear_form(oracle, p, deform):
    box = oracle.Box.make(coarse=(2, 2, 1), refine=1, hi=(2.0, 2.0, 1.0), deform=deform)
    plain, cons, idx = oracle.dofs(box, p)
    xq, _ = oracle.quadrature(box, p)
    kappa = np.exp(fourier_field(xq, seed=3))
    G = oracle.geometry_G(box, p, 0, kappa.reshape(-1))
    rng = np.random.default_rng(7)
    N = cons.shape[0]
    u, v = rng.uniform(-1, 1, N), rng.uniform(-1, 1, N)
    u[cons == 1] = 0.0
    v[cons == 1] = 0.0
    form = oracle.qp_form(p, idx, G, u, v)
    uAv = u @ oracle.vmult(p, idx, G, cons, v)
    assert abs(form.sum() - uAv) <= 1e-12 * np.abs(form).sum()
    # symmetry and alpha scaling
    assert np.allclose(oracle.qp_form(p, idx, G, v, u, -2.0), -2.0 * form, rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("nq_src,nq_dst,r_src,r_dst", [(5, 3, 2, 2), (5, 5, 2, 1), (3, 2, 2, 0), (4, 4, 1, 1)])
def test_coefficient_interpolation_exact_on_polynomial_logs(oracle, nq_src, nq_dst, r_src, r_dst):
    sb = oracle.Box.make(coarse=(2, 1, 1), refine=r_src, hi=(2.0, 1.0, 1.0))
    db = oracle.Box.make(coarse=(2, 1, 1), refine=r_dst, hi=(2.0, 1.0, 1.0))
    deg = nq_src - 1
    f = lambda x: 0.3 * x[..., 0] ** min(deg, 2) - 0.2 * x[..., 1] + 0.1 * x[..., 2] ** deg  # noqa: E731
    xs, _ = oracle.quadrature(sb, nq_src - 1, nq_src)
    xd, _ = oracle.quadrature(db, nq_dst - 1, nq_dst)
    out = oracle.coef_interpolate(sb, nq_src, np.exp(f(xs)), db, nq_dst)
    assert np.abs(np.log(out) - f(xd)).max() < 1e-12


def test_adjoint_gradient_matches_central_differences(oracle):
    """J(m) = 1/2 (u-u_d)^T M (u-u_d) on Q3, 4^3 cells; 3 directions, eps = 1e-6."""
    p = 3
    box = oracle.Box.make(refine=2)
    plain, cons, idx = oracle.dofs(box, p)
    xq, jxw = oracle.quadrature(box, p)
    b = oracle.rhs(box, p, p + 1, 0, plain, cons)

    def solve(m):
        G = oracle.geometry_G(box, p, 0, np.exp(m).reshape(-1))
        d = oracle.diagonal(p, idx, G, cons)
        return oracle.cg(lambda v: oracle.vmult(p, idx, G, cons, v), b, d, 1e-14), G

    def J_of(m):
        u, _ = solve(m)
        e = u - u_d
        return 0.5 * e @ oracle.mass_vmult(p, idx, jxw, cons, e)

    u_d, _ = solve(fourier_field(xq, seed=2))
    m = fourier_field(xq, seed=1)
    u, G = solve(m)
    e = u - u_d
    r = oracle.mass_vmult(p, idx, jxw, cons, e)
    d = oracle.diagonal(p, idx, G, cons)
    lam = oracle.cg(lambda v: oracle.vmult(p, idx, G, cons, v), r, d, 1e-14)
    g = oracle.qp_form(p, idx, G, lam, u, -1.0)
    eps = 1e-6
    for k in range(3):
        dm = fourier_field(xq, seed=100 + k)
        fd = (J_of(m + eps * dm) - J_of(m - eps * dm)) / (2 * eps)
        ad = float((g * dm).sum())
        assert abs(fd - ad) <= 1e-6 * abs(ad), (k, fd, ad)
