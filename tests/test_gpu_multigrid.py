"""Parity of the CUDA transfers, Chebyshev smoother, V-cycle and CG with the CPU oracle,
and of the whole mixed-precision solver with the reference's logged iteration counts."""
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def obox(oracle, b):
    return oracle.Box.make(coarse=tuple(b.coarse), refine=b.refine, lo=tuple(b.lo), hi=tuple(b.hi),
                           deform=b.deform, amp=b.amp, dirichlet_mask=b.dirichlet_mask)


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("pc,pf", [(1, 2), (2, 3), (3, 4), (2, 4), (3, 6), (1, 6)])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_p_transfer_matches_oracle(oracle, pc, pf, dtype):
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0))
    ob = obox(oracle, box)
    mesh = pmg.Mesh(box)
    oc, of = pmg.LaplaceOperator(mesh, pc, dtype), pmg.LaplaceOperator(mesh, pf, dtype)
    t = pmg.Transfer(oc, of)
    _, nc, nf = oracle.transfer_sizes(ob, pc, pf)
    rng = np.random.default_rng(pc * 10 + pf)
    xc, xf = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nf)
    base_f, base_c = rng.uniform(-1, 1, nf), rng.uniform(-1, 1, nc)
    tol = 1e-13 if dtype == pmg.F64 else 2e-6
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    ref = oracle.transfer_apply(ob, pc, pf, 0, xc, base_f.copy())
    d = torch.tensor(base_f, dtype=td, device="cuda")
    t.prolongate_and_add(d, torch.tensor(xc, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < tol
    ref = oracle.transfer_apply(ob, pc, pf, 1, xf, base_c.copy())
    d = torch.tensor(base_c, dtype=td, device="cuda")
    t.restrict_and_add(d, torch.tensor(xf, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < tol


@pytest.mark.parametrize("p", [1, 2, 4])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_h_transfer_matches_oracle(oracle, p, dtype):
    fine = pmg.Box.make(coarse=(2, 1, 1), refine=2, hi=(2.0, 1.0, 1.0))
    ob = obox(oracle, fine)
    oc = pmg.LaplaceOperator(pmg.Mesh(fine.with_refine(1)), p, dtype)
    of = pmg.LaplaceOperator(pmg.Mesh(fine), p, dtype)
    t = pmg.Transfer(oc, of)
    _, nc, nf = oracle.transfer_sizes(ob, p, p)
    rng = np.random.default_rng(p)
    xc, xf = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nf)
    tol = 1e-13 if dtype == pmg.F64 else 2e-6
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    ref = oracle.transfer_apply(ob, p, p, 0, xc, np.zeros(nf))
    d = torch.zeros(nf, dtype=td, device="cuda")
    t.prolongate_and_add(d, torch.tensor(xc, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < tol
    ref = oracle.transfer_apply(ob, p, p, 1, xf, np.zeros(nc))
    d = torch.zeros(nc, dtype=td, device="cuda")
    t.restrict_and_add(d, torch.tensor(xf, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < tol


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("degree,range_,eig_its", [(5, 15.0, 10), (0, 1e-3, 10000)])
def test_chebyshev_matches_oracle(oracle, mode, degree, range_, eig_its):
    box = pmg.Box.make(refine=2, deform=1)
    ob = obox(oracle, box)
    p = 2
    op = pmg.LaplaceOperator(pmg.Mesh(box), p, pmg.F64)
    n = op.m()
    eig = min(eig_its, n)
    sm = pmg.Chebyshev(op, degree, range_, eig)
    rng = np.random.default_rng(11)
    src, x0 = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    ref = x0.copy() if mode == 1 else np.zeros(n)
    mn, mx, deg = oracle.chebyshev_apply(ob, p, degree, range_, eig, mode, src, ref)
    d = torch.tensor(x0 if mode == 1 else np.zeros(n), device="cuda")
    s = torch.tensor(src, device="cuda")
    (sm.step if mode == 1 else sm.vmult)(d, s)
    torch.cuda.synchronize()
    info = sm.info()
    assert info["degree"] == deg
    assert abs(info["max_eigenvalue"] / mx - 1) < 1e-9 and abs(info["min_eigenvalue"] / mn - 1) < 1e-7
    assert rel_err(d.cpu().numpy(), ref) < 1e-10


with open(os.path.join(HERE, "golden", "reference_logs.json")) as f:
    LOGS = json.load(f)
CYCLES = {4: 1377, 5: 2601, 6: 4913, 7: 9537, 9: 35937, 10: 70785}


@pytest.mark.parametrize("cycle", sorted(CYCLES))
def test_fp64_multigrid_cg_matches_oracle_and_reference_log(oracle, cycle):
    box = pmg.doubling_box(cycle)
    ob = oracle.doubling_box(cycle)
    info_o, x_o = oracle.solve_box(ob, [4, 3, 2, 1], cheb=5, want_x=True)
    h = pmg.Hierarchy(box, [4, 3, 2, 1], mg_dtype=pmg.F64, cheb_degree=5)
    b = h.fine64.assemble_rhs(0)
    x, info = h.solve(b)
    torch.cuda.synchronize()
    assert info["iterations"] == info_o.iterations
    assert abs(info["reduction_per_step"] / info_o.reduction_per_step - 1) < 1e-6
    assert rel_err(x.cpu().numpy(), x_o) < 1e-8
    row = [r for r in LOGS["tables"]["fp64"] if r["dofs"] == CYCLES[cycle]][0]
    assert info["iterations"] == row["cg_its"]


@pytest.mark.parametrize("cycle", sorted(CYCLES))
def test_mixed_precision_multigrid_matches_reference_log(oracle, cycle):
    """FP32 V-cycle inside FP64 CG (the reference's mixed-precision configuration)."""
    box = pmg.doubling_box(cycle)
    h = pmg.Hierarchy(box, [4, 3, 2, 1], mg_dtype=pmg.F32, cheb_degree=5)
    b = h.fine64.assemble_rhs(0)
    x, info = h.solve(b)
    row = [r for r in LOGS["tables"]["mixed"] if r["dofs"] == CYCLES[cycle]][0]
    assert info["iterations"] == row["cg_its"]
    assert abs(info["reduction_per_step"] / row["cg_reduction"] - 1) < 0.03


def test_jacobi_cg_converges_on_deformed_mesh(oracle):
    box = pmg.Box.make(refine=2, deform=1)
    op = pmg.LaplaceOperator(pmg.Mesh(box), 3, pmg.F64)
    b = op.assemble_rhs(1, 5)
    x = op.initialize_dof_vector()
    info = pmg.solve_cg(op, x, b, None, reduce=1e-10, max_iterations=2000)
    assert info["converged"]
    r = op.initialize_dof_vector()
    op.vmult(r, x)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(r - b) / torch.linalg.norm(b)) < 1.1e-10


def test_cg_iteration_limit_reports_noconv():
    box = pmg.Box.make(refine=2)
    op = pmg.LaplaceOperator(pmg.Mesh(box), 2, pmg.F64)
    b = op.assemble_rhs(0)
    x = op.initialize_dof_vector()
    with pytest.raises(pmg.PmgError) as e:
        pmg.solve_cg(op, x, b, None, reduce=1e-12, max_iterations=2)
    assert e.value.status == -5


@pytest.mark.parametrize("mg_dtype", [pmg.F64, pmg.F32])
def test_variable_kappa_q6_phmg_matches_oracle(oracle, mg_dtype):
    """Q6 with kappa = 1 + 0.9 sin(2 pi x) sin(2 pi y) sin(2 pi z) on 3^3 coarse cells refined
    once (the variable-coefficient ph-multigrid configuration at a small size), affine
    geometry with the coefficient per quadrature point, solved to 1e-10."""
    box = pmg.Box.make(coarse=(3, 3, 3), refine=1)
    ob = oracle.Box.make(coarse=(3, 3, 3), refine=1)
    info_o, x_o = oracle.solve_box(ob, [6, 3, 2, 1], cheb=4, coeff_kind=1, reduce=1e-10, want_x=True)
    h = pmg.Hierarchy(box, [6, 3, 2, 1], mg_dtype=mg_dtype, cheb_degree=4,
                      geometry=pmg.GEOMETRY_AFFINE, coeff_kind=pmg.COEFF_KAPPA)
    x, info = h.solve(h.fine64.assemble_rhs(0), reduce=1e-10)
    torch.cuda.synchronize()
    assert info["converged"]
    assert abs(info["iterations"] - info_o.iterations) <= (0 if mg_dtype == pmg.F64 else 1)
    assert rel_err(x.cpu().numpy(), x_o) < 1e-8


@pytest.mark.parametrize("mg_dtype", [pmg.F64, pmg.F32])
def test_plain_q2_h_multigrid_matches_oracle(oracle, mg_dtype):
    """The plain method: -lap u = 3 pi^2 sin(pi x) sin(pi y) sin(pi z) on [0,1]^3 with FE_Q(2) on
    16^3 cells, geometric multigrid at degree 2 on every level (16^3 -> 8^3 -> 4^3 -> 2^3,
    GeometricTransfer<dim, fe_degree> as in source/geometric_multigrid/program.cc:245-249),
    Chebyshev(3), FP64 CG to 1e-10.  The FP64 V-cycle takes the oracle's iterations and
    solution; the FP32 V-cycle converges within one iteration of it."""
    box = pmg.Box.make(coarse=(2, 2, 2), refine=3)
    ob = oracle.Box.make(coarse=(2, 2, 2), refine=3)
    info_o, x_o = oracle.solve_box(ob, [2], cheb=3, rhs_kind=1, reduce=1e-10, want_x=True, h_degree=2)
    h = pmg.Hierarchy(box, [2], mg_dtype=mg_dtype, cheb_degree=3, h_degree=2)
    assert [lv.degree for lv in h.levels] == [2, 2, 2, 2]
    assert [lv.n_cells() for lv in h.levels] == [8, 64, 512, 4096]
    b = h.fine64.assemble_rhs(1, 4)
    x, info = h.solve(b, reduce=1e-10)
    torch.cuda.synchronize()
    assert h.fine64.m() == info_o.n_dofs == 35937
    assert info["converged"]
    if mg_dtype == pmg.F64:
        assert info["iterations"] == info_o.iterations
        assert abs(info["reduction_per_step"] / info_o.reduction_per_step - 1) < 1e-6
    else:
        assert abs(info["iterations"] - info_o.iterations) <= 1
    assert rel_err(x.cpu().numpy(), x_o) < 1e-8
    assert abs(h.fine64.l2_error(x, 1) / info_o.l2_error - 1) < 1e-6


def test_plain_q2_h_multigrid_converges_at_rate_three():
    """L2 error of the config-1 solve on 8^3, 16^3, 32^3 cells falls like h^3 (FE_Q(2))."""
    errs = []
    for refine in (2, 3, 4):
        h = pmg.Hierarchy(pmg.Box.make(coarse=(2, 2, 2), refine=refine), [2], mg_dtype=pmg.F32,
                          cheb_degree=3, h_degree=2)
        x, info = h.solve(h.fine64.assemble_rhs(1, 4), reduce=1e-10)
        assert info["converged"] and info["iterations"] <= 8
        errs.append(h.fine64.l2_error(x, 1))
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(2.85 < r < 3.15 for r in rates), rates


def test_plain_q6_kappa_h_multigrid_matches_oracle(oracle):
    """The plain method on the variable-coefficient Q6 problem: FE_Q(6) on every level (3^3 and
    6^3 cells, kappa = 1 + 0.9 sin(2 pi x) sin(2 pi y) sin(2 pi z)), the (2p+1)-node h-transfer
    at p = 6, Chebyshev(4), FP64 throughout: the oracle's iterations and solution."""
    box = pmg.Box.make(coarse=(3, 3, 3), refine=1)
    ob = oracle.Box.make(coarse=(3, 3, 3), refine=1)
    info_o, x_o = oracle.solve_box(ob, [6], cheb=4, coeff_kind=1, reduce=1e-10, want_x=True, h_degree=6)
    h = pmg.Hierarchy(box, [6], mg_dtype=pmg.F64, cheb_degree=4, h_degree=6, geometry=pmg.GEOMETRY_AFFINE,
                      coeff_kind=pmg.COEFF_KAPPA)
    x, info = h.solve(h.fine64.assemble_rhs(0), reduce=1e-10)
    torch.cuda.synchronize()
    assert info["converged"] and info["iterations"] == info_o.iterations
    assert rel_err(x.cpu().numpy(), x_o) < 1e-8


@pytest.mark.parametrize("mode", [1, 3])
def test_variable_kappa_q6_phmg_with_tensor_core_levels(oracle, mode):
    """The FP32 V-cycle with its affine levels on the tensor cores (TF32 or three TF32
    products) inside FP64 CG: converges to 1e-10 within one iteration of the oracle's count and
    gives its solution to 1e-8."""
    box = pmg.Box.make(coarse=(3, 3, 3), refine=1)
    ob = oracle.Box.make(coarse=(3, 3, 3), refine=1)
    info_o, x_o = oracle.solve_box(ob, [6, 3, 2, 1], cheb=4, coeff_kind=1, reduce=1e-10, want_x=True)
    h = pmg.Hierarchy(box, [6, 3, 2, 1], mg_dtype=pmg.F32, cheb_degree=4, geometry=pmg.GEOMETRY_AFFINE,
                      coeff_kind=pmg.COEFF_KAPPA, tensor_cores=mode)
    x, info = h.solve(h.fine64.assemble_rhs(0), reduce=1e-10)
    torch.cuda.synchronize()
    assert info["converged"]
    assert abs(info["iterations"] - info_o.iterations) <= 1
    assert rel_err(x.cpu().numpy(), x_o) < 1e-8
