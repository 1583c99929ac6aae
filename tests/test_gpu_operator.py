"""Parity of the CUDA level operator (vmult, diagonal, index map, geometry, right-hand
side) with the CPU oracle, called through the C ABI.

Tolerances: FP64 kernels agree with the FP64 oracle to 1e-12 relative (max-norm of the
difference over the max-norm of the result); FP32 kernels to 2e-5 relative."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = {pmg.F64: 1e-12, pmg.F32: 2e-5}


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def tdtype(dt):
    return torch.float64 if dt == pmg.F64 else torch.float32


def obox(oracle, b):
    return oracle.Box.make(coarse=tuple(b.coarse), refine=b.refine, lo=tuple(b.lo), hi=tuple(b.hi),
                           deform=b.deform, amp=b.amp, dirichlet_mask=b.dirichlet_mask)


def random_src(n, seed=1234):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n)


BOXES = {
    "unit_r2": dict(refine=2),
    "deformed_r2": dict(refine=2, deform=1),
    "ragged_3x2x1": dict(coarse=(3, 2, 1), refine=1, hi=(3.0, 2.0, 1.0)),
    "single_cell": dict(refine=0),
}


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("boxname", list(BOXES))
def test_vmult_matches_oracle(oracle, degree, dtype, boxname):
    box = pmg.Box.make(**BOXES[boxname])
    ob = obox(oracle, box)
    mesh = pmg.Mesh(box)
    op = pmg.LaplaceOperator(mesh, degree, dtype)
    plain, cons, idx = oracle.dofs(ob, degree)
    assert op.m() == cons.shape[0]
    np.testing.assert_array_equal(op.dof_indices(), idx)
    np.testing.assert_array_equal(op.constrained(), cons)
    G = oracle.geometry_G(ob, degree)
    src = random_src(op.m())
    ref = oracle.vmult(degree, idx, G, cons, src)
    s = torch.tensor(src, dtype=tdtype(dtype), device="cuda")
    d = op.initialize_dof_vector()
    op.vmult(d, s)
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype]


@pytest.mark.parametrize("degree", [2, 4])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_full_and_affine_geometry_agree_and_kappa(oracle, degree, dtype):
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0))
    ob = obox(oracle, box)
    mesh = pmg.Mesh(box)
    plain, cons, idx = oracle.dofs(ob, degree)
    src = random_src(cons.shape[0], 7)
    s = torch.tensor(src, dtype=tdtype(dtype), device="cuda")
    for kind in (pmg.COEFF_NONE, pmg.COEFF_KAPPA):
        ref = oracle.vmult(degree, idx, oracle.geometry_G(ob, degree, coeff_kind=kind), cons, src)
        for geom in (pmg.GEOMETRY_FULL, pmg.GEOMETRY_AFFINE):
            op = pmg.LaplaceOperator(mesh, degree, dtype, geom, kind)
            d = op.initialize_dof_vector()
            op.vmult(d, s)
            torch.cuda.synchronize()
            assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype], (kind, geom)


def test_coefficient_values_per_point(oracle):
    degree = 3
    box = pmg.Box.make(refine=1, deform=1)
    ob = obox(oracle, box)
    mesh = pmg.Mesh(box)
    C = box.ncells()
    kap = np.exp(np.random.default_rng(5).normal(0, 0.5, (C, (degree + 1) ** 3)))
    plain, cons, idx = oracle.dofs(ob, degree)
    ref_G = oracle.geometry_G(ob, degree, kappa_qp=kap)
    op = pmg.LaplaceOperator(mesh, degree, pmg.F64, pmg.GEOMETRY_FULL, pmg.COEFF_VALUES, kap)
    assert rel_err(op.geometry(), ref_G) < 1e-13
    src = random_src(op.m(), 3)
    d = op.initialize_dof_vector()
    op.vmult(d, torch.tensor(src, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.cpu().numpy(), oracle.vmult(degree, idx, ref_G, cons, src)) < 1e-12


@pytest.mark.parametrize("degree", [1, 4, 6])
def test_geometry_tensor_matches_oracle(oracle, degree):
    box = pmg.Box.make(refine=1, deform=1, amp=0.1)
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, pmg.F64, pmg.GEOMETRY_FULL)
    assert rel_err(op.geometry(), oracle.geometry_G(ob, degree)) < 1e-13


@pytest.mark.parametrize("degree", [1, 2, 4, 6])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("deform", [0, 1])
def test_diagonal_matches_oracle(oracle, degree, dtype, deform):
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0), deform=deform)
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, dtype)
    plain, cons, idx = oracle.dofs(ob, degree)
    ref = oracle.diagonal(degree, idx, oracle.geometry_G(ob, degree), cons)
    op.compute_diagonal()
    inv = op.get_matrix_diagonal_inverse()
    torch.cuda.synchronize()
    assert rel_err(1.0 / inv.double().cpu().numpy(), ref) < TOL[dtype] * 10
    i = int(np.argmax(cons == 0))
    assert abs(op.el(i, i) / ref[i] - 1) < TOL[dtype] * 10


@pytest.mark.parametrize("f_kind,nq", [(0, 0), (1, 6)])
def test_rhs_matches_oracle(oracle, f_kind, nq):
    degree = 4
    box = pmg.Box.make(refine=2, deform=1)
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, pmg.F64)
    plain, cons, idx = oracle.dofs(ob, degree)
    ref = oracle.rhs(ob, degree, nq if nq else degree + 1, f_kind, plain, cons)
    b = op.assemble_rhs(f_kind, nq)
    torch.cuda.synchronize()
    assert rel_err(b.cpu().numpy(), ref) < 1e-13


def test_vmult_dummy_and_tvmult(oracle):
    box = pmg.Box.make(refine=1)
    op = pmg.LaplaceOperator(pmg.Mesh(box), 3, pmg.F64)
    src = torch.tensor(random_src(op.m()), device="cuda")
    a, b, c = (op.initialize_dof_vector() for _ in range(3))
    op.vmult(a, src)
    op.Tvmult(b, src)
    op.vmult_dummy(c, src, True, True)
    torch.cuda.synchronize()
    assert torch.equal(a, b) or rel_err(a.cpu().numpy(), b.cpu().numpy()) < 1e-15
    assert rel_err(c.cpu().numpy(), a.cpu().numpy()) < 1e-15
    op.vmult_dummy(c, src, True, False)
    torch.cuda.synchronize()
    cons = torch.tensor(op.constrained(), device="cuda").bool()
    assert torch.all(c[~cons] == 0) and torch.equal(c[cons], src[cons])


def test_invalid_arguments_raise():
    mesh = pmg.Mesh(pmg.Box.make(refine=0))
    with pytest.raises(pmg.PmgError) as e:
        pmg.LaplaceOperator(mesh, 7)
    assert e.value.status == -1
    op = pmg.LaplaceOperator(mesh, 2)
    with pytest.raises(pmg.PmgError) as e:
        op.get_matrix_diagonal_inverse()
    assert e.value.status == -7
    v = op.initialize_dof_vector()
    with pytest.raises(pmg.PmgError):
        op.vmult(v, v)  # aliasing is rejected


@pytest.mark.parametrize("degree", [1, 2, 4, 6])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("boxname", ["unit_r2", "deformed_r2", "ragged_3x2x1"])
def test_l2_error_matches_oracle(oracle, degree, dtype, boxname):
    """||u_h - sin sin sin||_L2 on the GPU against the oracle's host loop, every DoF's value
    counted (Dirichlet ones included)."""
    box = pmg.Box.make(**BOXES[boxname])
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, dtype)
    plain, cons, idx = oracle.dofs(ob, degree)
    u = random_src(op.m(), 7)
    ut = torch.tensor(u, dtype=tdtype(dtype), device="cuda")
    u_used = ut.double().cpu().numpy()  # the values the GPU sees (rounded in FP32)
    for nq in (degree + 1, degree + 2):
        got = op.l2_error(ut, 1, nq)
        want = oracle.l2_error_sine(ob, degree, nq, plain, u_used)
        assert abs(got - want) <= 1e-12 * want


# ---- the deal.II-style formulation (PMG_GEOMETRY_INVJAC: J^{-1} and JxW per point) ----

@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("boxname,kind", [("deformed_r2", pmg.COEFF_NONE), ("ragged_3x2x1", pmg.COEFF_NONE),
                                          ("deformed_r2", pmg.COEFF_KAPPA), ("single_cell", pmg.COEFF_NONE)])
def test_invjac_vmult_matches_oracle_invjac(oracle, degree, dtype, boxname, kind):
    """The inverse-Jacobian formulation on the GPU against the oracle's restatement of
    portable_local_laplace_operator.h:329-347 (orc_vmult_invjac)."""
    box = pmg.Box.make(**BOXES[boxname])
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, dtype, pmg.GEOMETRY_INVJAC, kind)
    plain, cons, idx = oracle.dofs(ob, degree)
    iJ, jxw = oracle.invjac(ob, degree, coeff_kind=kind)
    src = random_src(op.m(), 11)
    ref = oracle.vmult_invjac(degree, idx, iJ, jxw, cons, src)
    s = torch.tensor(src, dtype=tdtype(dtype), device="cuda")
    d = op.initialize_dof_vector()
    op.vmult(d, s)
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype]
    # the same operator as the G formulation
    ref_g = oracle.vmult(degree, idx, oracle.geometry_G(ob, degree, coeff_kind=kind), cons, src)
    assert rel_err(d.double().cpu().numpy(), ref_g) < TOL[dtype]


@pytest.mark.parametrize("degree", [2, 4, 6])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_invjac_diagonal_matches_oracle(oracle, degree, dtype):
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0), deform=1)
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, dtype, pmg.GEOMETRY_INVJAC)
    plain, cons, idx = oracle.dofs(ob, degree)
    ref = oracle.diagonal(degree, idx, oracle.geometry_G(ob, degree), cons)
    op.compute_diagonal()
    inv = op.get_matrix_diagonal_inverse()
    torch.cuda.synchronize()
    assert rel_err(1.0 / inv.double().cpu().numpy(), ref) < TOL[dtype] * 10


def test_invjac_multigrid_solve_matches_g_formulation():
    """A Q4 ph-multigrid CG solve on the deformed cube with every level in the inverse-Jacobian
    formulation takes the iterations of the G formulation and reaches the same solution."""
    box = pmg.Box.make(refine=3, deform=1)
    res = {}
    for geom in (pmg.GEOMETRY_FULL, pmg.GEOMETRY_INVJAC):
        h = pmg.Hierarchy(box, [4, 2, 1], mg_dtype=pmg.F32, cheb_degree=4, geometry=geom)
        b = h.fine64.assemble_rhs(1)
        h.estimate()
        x, info = h.solve(b, reduce=1e-10)
        res[geom] = (x.cpu().numpy(), info["iterations"])
    assert res[pmg.GEOMETRY_INVJAC][1] == res[pmg.GEOMETRY_FULL][1]
    assert rel_err(res[pmg.GEOMETRY_INVJAC][0], res[pmg.GEOMETRY_FULL][0]) < 1e-9


def test_invjac_rejects_the_per_point_form():
    op = pmg.LaplaceOperator(pmg.Mesh(pmg.Box.make(refine=1)), 2, pmg.F64, pmg.GEOMETRY_INVJAC)
    u = torch.zeros(op.m(), dtype=torch.float64, device="cuda")
    with pytest.raises(pmg.PmgError):
        op.qp_form(u, u, 1.0)


@pytest.mark.parametrize("degree", [3, 5])
def test_invjac_coefficient_values_and_update_match_g(degree):
    """Per-point coefficient values folded into JxW (and replaced later) give the operator of
    the G formulation with the same values."""
    box = pmg.Box.make(refine=2, deform=1)
    mesh = pmg.Mesh(box)
    nq3 = (degree + 1) ** 3
    rng = np.random.default_rng(degree)
    k1 = np.exp(rng.uniform(-0.5, 0.5, (mesh.n_cells(), nq3)))
    k2 = np.exp(rng.uniform(-0.5, 0.5, (mesh.n_cells(), nq3)))
    ops = [pmg.LaplaceOperator(mesh, degree, pmg.F64, g, pmg.COEFF_VALUES, k1)
           for g in (pmg.GEOMETRY_FULL, pmg.GEOMETRY_INVJAC)]
    s = torch.tensor(random_src(ops[0].m(), 5), dtype=torch.float64, device="cuda")
    for values in (None, k2):
        out = []
        for op in ops:
            if values is not None:
                op.set_coefficient(values)
            d = op.initialize_dof_vector()
            op.vmult(d, s)
            out.append(d.cpu().numpy())
        torch.cuda.synchronize()
        assert rel_err(out[1], out[0]) < 1e-12


@pytest.mark.parametrize("mask", [0x00, 0x13])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_subdomain_operator_with_neumann_faces(oracle, mask, dtype):
    """The operator of a subdomain with Neumann faces (the SubdomainLaplaceOperator the
    reference's BNN preconditioner solves with, include/domain_decomposition/
    portable_bnn_preconditioner.h:146-277): the same cell kernel on a box whose faces outside
    dirichlet_mask carry no constraints.  Matches the oracle; a floating subdomain (no
    Dirichlet face) maps the constant vector to zero."""
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0), deform=1, dirichlet_mask=mask)
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), 3, dtype)
    plain, cons, idx = oracle.dofs(ob, 3)
    assert int(cons.sum()) == int(op.constrained().sum()) and (mask != 0 or cons.sum() == 0)
    src = random_src(op.m(), 21)
    ref = oracle.vmult(3, idx, oracle.geometry_G(ob, 3), cons, src)
    d = op.initialize_dof_vector()
    op.vmult(d, torch.tensor(src, dtype=tdtype(dtype), device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype]
    if mask == 0:
        one = torch.ones(op.m(), dtype=tdtype(dtype), device="cuda")
        op.vmult(d, one)
        torch.cuda.synchronize()
        scale = float(np.abs(ref).max())
        assert float(d.abs().max()) < (1e-12 if dtype == pmg.F64 else 1e-5) * scale


# the tensor-core cell kernel: TF32 products (mode 1, 10-bit mantissas) and three TF32 products
# (mode 3, about FP32 accuracy), against the FP64 oracle
TC_TOL = {1: 5e-3, 3: 2e-5}


@pytest.mark.parametrize("mode", [1, 3])
@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("coeff", [pmg.COEFF_NONE, pmg.COEFF_KAPPA])
def test_tensor_core_vmult_matches_oracle(oracle, mode, degree, coeff):
    box = pmg.Box.make(coarse=(3, 2, 2), refine=1, hi=(3.0, 2.0, 2.0))
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, pmg.F32, pmg.GEOMETRY_AFFINE, coeff)
    op.set_tensor_cores(mode)
    plain, cons, idx = oracle.dofs(ob, degree)
    src = random_src(op.m(), 5)
    ref = oracle.vmult(degree, idx, oracle.geometry_G(ob, degree, coeff_kind=coeff), cons, src)
    d = op.initialize_dof_vector()
    op.vmult(d, torch.tensor(src, dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TC_TOL[mode]


@pytest.mark.parametrize("mode", [1, 3])
def test_tensor_core_vmult_many_cells_per_warp(oracle, mode):
    """Q6 with kappa on 24^3 cells (the config-3 fine level at a smaller size): every warp
    applies several cells."""
    box = pmg.Box.make(coarse=(3, 3, 3), refine=3)
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), 6, pmg.F32, pmg.GEOMETRY_AFFINE, pmg.COEFF_KAPPA)
    op.set_tensor_cores(mode)
    plain, cons, idx = oracle.dofs(ob, 6)
    src = random_src(op.m(), 6)
    ref = oracle.vmult(6, idx, oracle.geometry_G(ob, 6, coeff_kind=pmg.COEFF_KAPPA), cons, src)
    d = op.initialize_dof_vector()
    op.vmult(d, torch.tensor(src, dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    units, par = op.last_launch()
    assert units >= 2 * par
    assert rel_err(d.double().cpu().numpy(), ref) < TC_TOL[mode]


def test_tensor_core_mode_rejected_where_not_built():
    op = pmg.LaplaceOperator(pmg.Mesh(pmg.Box.make(refine=1, deform=1)), 2, pmg.F32, pmg.GEOMETRY_FULL)
    with pytest.raises(pmg.PmgError):
        op.set_tensor_cores(1)
    op64 = pmg.LaplaceOperator(pmg.Mesh(pmg.Box.make(refine=1)), 2, pmg.F64, pmg.GEOMETRY_AFFINE)
    with pytest.raises(pmg.PmgError):
        op64.set_tensor_cores(3)


# cell ranges (pmg_operator_vmult_cells): the split of a sharded vmult into the cells computed
# while the ghost update is in flight and the rest; the sum of the passes equals vmult up to
# the order of the additions, and the oracle on the same cells
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("degree,geometry,coeff", [(3, pmg.GEOMETRY_FULL, pmg.COEFF_NONE),
                                                   (4, pmg.GEOMETRY_FULL, pmg.COEFF_NONE),
                                                   (2, pmg.GEOMETRY_AFFINE, pmg.COEFF_KAPPA),
                                                   (5, pmg.GEOMETRY_INVJAC, pmg.COEFF_NONE)])
def test_vmult_cells_passes_sum_to_vmult(oracle, dtype, degree, geometry, coeff):
    box = pmg.Box.make(coarse=(3, 2, 2), refine=2, hi=(3.0, 2.0, 2.0),
                       deform=0 if geometry == pmg.GEOMETRY_AFFINE else 1)
    ob = obox(oracle, box)
    op = pmg.LaplaceOperator(pmg.Mesh(box), degree, dtype, geometry, coeff)
    cpw = op.cells_per_group()
    assert cpw == 32 // (degree + 1)
    n_cells = op.n_cells()
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    src = torch.tensor(random_src(op.m(), 3), dtype=td, device="cuda")
    full = op.initialize_dof_vector()
    op.vmult(full, src)
    cut1 = (n_cells // 3 // cpw) * cpw
    cut2 = (2 * n_cells // 3 // cpw) * cpw
    for cuts in ([0, n_cells], [0, cut1, n_cells], [0, cut1, cut2, n_cells], [0, 0, n_cells]):
        d = torch.full_like(full, 7.0)  # overwritten by the first (init) pass
        for k, (a, b) in enumerate(zip(cuts, cuts[1:])):
            op.vmult_cells(d, src, a, b, k == 0)
        torch.cuda.synchronize()
        assert rel_err(d.double().cpu().numpy(), full.double().cpu().numpy()) < (1e-14 if dtype == pmg.F64 else 1e-6)
    # one pass over a range alone against the oracle on those cells (plus the identity rows)
    plain, cons, idx = oracle.dofs(ob, degree)
    if geometry == pmg.GEOMETRY_INVJAC:
        iJ, jxw = oracle.invjac(ob, degree, coeff)
        ref = oracle.vmult_invjac(degree, idx[cut1:], np.ascontiguousarray(iJ.reshape(n_cells, -1)[cut1:]).reshape(-1),
                                  np.ascontiguousarray(jxw.reshape(n_cells, -1)[cut1:]).reshape(-1), cons,
                                  src.double().cpu().numpy())
    else:
        G = oracle.geometry_G(ob, degree, coeff_kind=coeff).reshape(n_cells, -1)
        ref = oracle.vmult(degree, idx[cut1:], G[cut1:], cons, src.double().cpu().numpy())
    d = op.initialize_dof_vector()
    op.vmult_cells(d, src, cut1, n_cells, True)
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype]


def test_vmult_cells_rejects_bad_ranges():
    op = pmg.LaplaceOperator(pmg.Mesh(pmg.Box.make(refine=2, deform=1)), 4, pmg.F64)
    cpw = op.cells_per_group()
    src = torch.zeros(op.m(), dtype=torch.float64, device="cuda")
    dst = torch.zeros_like(src)
    for a, b in ((1, cpw * 2), (0, cpw + 1), (cpw * 2, cpw), (-cpw, 0), (0, 65)):
        with pytest.raises(pmg.PmgError):
            op.vmult_cells(dst, src, a, b, True)
    op.vmult_cells(dst, src, 0, 64, True)  # the cell count ends a range anywhere
    dg = pmg.DGLaplaceOperator(pmg.Mesh(pmg.Box.make(refine=1)), 2, pmg.F64)
    v = torch.zeros(dg.m(), dtype=torch.float64, device="cuda")
    with pytest.raises(pmg.PmgError):
        dg.vmult_cells(v, v.clone(), 0, 8, True)
