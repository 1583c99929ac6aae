"""Parity with the CPU oracle at sizes where every warp of a grid-stride kernel processes two
or more work units (warp groups of cells, cell batches, transfer patches).

The kernels launch at most one grid of resident warps and loop over the groups
(`for g = warp0; g < n_groups; g += nwarps`).  Only the second and later trips of that loop
exercise what carries state from one group to the next: the geometry ring refilled from the
next group's first column, the mbarrier phase carried across groups, the one-group-ahead
index pipeline, the L2 prefetch of the next group.  Every case below asserts, from the shape
of the launch the library reports (pmg_operator_last_launch / pmg_transfer_last_launch),
that units >= 2 * parallel, and then compares with the oracle (FP64 to 1e-12, FP32 to 2e-5
relative in the max norm, as in the small-mesh tests)."""
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


def assert_multi_unit(shape):
    units, par = shape
    assert par > 0 and units >= 2 * par, f"{units} units over {par} warps: not every warp takes two"


def apply(op, src, dtype):
    d = op.initialize_dof_vector()
    op.vmult(d, torch.tensor(src, dtype=tdtype(dtype), device="cuda"))
    torch.cuda.synchronize()
    return d.double().cpu().numpy()


# (name, box, degree, geometry, coefficient): Q4 on the deformed 32^3 cube (the benchmark's
# mesh family; FP64 runs the geometry-ring variant), Q5 full geometry (FP64: ring plus the
# index pipeline), Q6 affine with kappa on 24^3 (the config-3 fine level; FP32: index
# pipeline), and the inverse-Jacobian formulation on the deformed 32^3 cube
CASES = [
    ("q4_deformed_32", dict(refine=5, deform=1), 4, pmg.GEOMETRY_FULL, pmg.COEFF_NONE),
    ("q5_deformed_24", dict(coarse=(3, 3, 3), refine=3, deform=1), 5, pmg.GEOMETRY_FULL, pmg.COEFF_NONE),
    ("q6_affine_kappa_24", dict(coarse=(3, 3, 3), refine=3), 6, pmg.GEOMETRY_AFFINE, pmg.COEFF_KAPPA),
    ("q4_invjac_32", dict(refine=5, deform=1), 4, pmg.GEOMETRY_INVJAC, pmg.COEFF_NONE),
    # Q2 on the deformed 64^3 cube (FP64: ring with the index pipeline) and Q3 on 64^3 (FP64:
    # ring with the register pipeline)
    ("q2_deformed_64", dict(refine=6, deform=1), 2, pmg.GEOMETRY_FULL, pmg.COEFF_NONE),
    ("q3_deformed_64", dict(refine=6, deform=1), 3, pmg.GEOMETRY_FULL, pmg.COEFF_NONE),
    # Q6 full geometry on the deformed 24^3 cube (FP32: ring; FP64: direct loads with the L2
    # prefetch of the next group)
    ("q6_deformed_24", dict(coarse=(3, 3, 3), refine=3, deform=1), 6, pmg.GEOMETRY_FULL, pmg.COEFF_NONE),
]


@pytest.fixture(scope="module")
def problems(oracle):
    """Oracle index maps and reference results per case, shared by both dtypes."""
    out = {}
    for name, bkw, p, geometry, coeff in CASES:
        box = pmg.Box.make(**bkw)
        ob = obox(oracle, box)
        plain, cons, idx = oracle.dofs(ob, p)
        src = np.random.default_rng(1234).uniform(-1.0, 1.0, cons.shape[0])
        if geometry == pmg.GEOMETRY_INVJAC:
            iJ, jxw = oracle.invjac(ob, p, coeff)
            ref = oracle.vmult_invjac(p, idx, iJ, jxw, cons, src)
        else:
            ref = oracle.vmult(p, idx, oracle.geometry_G(ob, p, coeff_kind=coeff), cons, src)
        out[name] = (box, idx, src, ref)
    return out


@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("case", [c[0] for c in CASES])
def test_vmult_multi_group_matches_oracle(problems, case, dtype):
    _, _, p, geometry, coeff = next(c for c in CASES if c[0] == case)
    box, idx, src, ref = problems[case]
    op = pmg.LaplaceOperator(pmg.Mesh(box), p, dtype, geometry, coeff)
    got = apply(op, src, dtype)
    assert_multi_unit(op.last_launch(pmg.KERNEL_VMULT_CELL))
    assert rel_err(got, ref) < TOL[dtype]
    # a second launch (the mbarriers and rings start afresh) gives the same result
    assert rel_err(apply(op, src, dtype), ref) < TOL[dtype]
    if dtype == pmg.F64:
        np.testing.assert_array_equal(op.dof_indices(), idx)


@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("kind,p_c,p_f,refine,multi", [("p", 2, 4, 5, True), ("p", 3, 6, 4, False),
                                                       ("h", 1, 1, 6, True), ("h", 2, 2, 6, True)])
def test_transfer_multi_patch_matches_oracle(oracle, kind, p_c, p_f, refine, multi, dtype):
    """p-transfers on the 32^3 mesh (one patch per cell) and h-transfers onto the 64^3 fine
    mesh (one patch per coarse 32^3 cell), every warp taking two or more patches; Q3 -> Q6 on
    16^3 cells (fewer patches than resident warps: the oracle's Q6 levels at 32^3 take minutes)
    for parity only."""
    fine = pmg.Box.make(refine=refine)
    ob = obox(oracle, fine)
    if kind == "p":
        mesh = pmg.Mesh(fine)
        oc, of = pmg.LaplaceOperator(mesh, p_c, dtype), pmg.LaplaceOperator(mesh, p_f, dtype)
    else:
        oc = pmg.LaplaceOperator(pmg.Mesh(fine.with_refine(refine - 1)), p_c, dtype)
        of = pmg.LaplaceOperator(pmg.Mesh(fine), p_f, dtype)
    t = pmg.Transfer(oc, of)
    _, nc, nf = oracle.transfer_sizes(ob, p_c, p_f)
    rng = np.random.default_rng(17)
    xc, xf = rng.uniform(-1, 1, nc), rng.uniform(-1, 1, nf)
    base_f, base_c = rng.uniform(-1, 1, nf), rng.uniform(-1, 1, nc)
    tol = 1e-13 if dtype == pmg.F64 else 2e-6
    td = tdtype(dtype)
    ref = oracle.transfer_apply(ob, p_c, p_f, 0, xc, base_f.copy())
    d = torch.tensor(base_f, dtype=td, device="cuda")
    t.prolongate_and_add(d, torch.tensor(xc, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    if multi:
        assert_multi_unit(t.last_launch())
    assert rel_err(d.double().cpu().numpy(), ref) < tol
    ref = oracle.transfer_apply(ob, p_c, p_f, 1, xf, base_c.copy())
    d = torch.tensor(base_c, dtype=td, device="cuda")
    t.restrict_and_add(d, torch.tensor(xf, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    if multi:
        assert_multi_unit(t.last_launch())
    assert rel_err(d.double().cpu().numpy(), ref) < tol


@pytest.fixture(scope="module")
def dg_problem(oracle):
    """DG-SIPG Q3 on 64^3 cells (16,777,216 DoFs, 4096 tiles of 4x4x4 cells) and the
    oracle's result, shared by both dtypes."""
    p = 3
    box = pmg.Box.make(coarse=(2, 2, 2), refine=5)
    c_pen = 2.0 * (p + 1) ** 2
    ob = obox(oracle, box)
    src = np.random.default_rng(p).uniform(-1, 1, oracle.dg_n(ob, p))
    return p, box, c_pen, src, oracle.dg_vmult(ob, p, c_pen, src)


@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_dg_vmult_multi_batch_matches_oracle(dg_problem, dtype):
    """The face kernel loops over 4x4x4 cell tiles (every block takes two or more), the cell
    kernel over warp groups."""
    p, box, c_pen, src, ref = dg_problem
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype, c_pen)
    got = apply(op, src, dtype)
    assert_multi_unit(op.last_launch(pmg.KERNEL_DG_FACES))
    assert_multi_unit(op.last_launch(pmg.KERNEL_VMULT_CELL))
    assert rel_err(got, ref) < TOL[dtype]


@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_mass_and_qp_form_multi_group_match_oracle(oracle, dtype):
    """Mass matrix (per-point weights with a coefficient) and the per-point form on the
    deformed 64^3 cube at Q2 (26,215 warp groups)."""
    from pmg.adjoint import fourier_field
    p = 2
    box = pmg.Box.make(refine=6, deform=1)
    ob = obox(oracle, box)
    plain, cons, idx = oracle.dofs(ob, p)
    xq, jxw = oracle.quadrature(ob, p)
    kappa = np.exp(fourier_field(xq, seed=11))
    mesh = pmg.Mesh(box)
    rng = np.random.default_rng(5)
    u, v = rng.uniform(-1, 1, cons.shape[0]), rng.uniform(-1, 1, cons.shape[0])
    M = pmg.MassOperator(mesh, p, dtype, pmg.GEOMETRY_FULL, pmg.COEFF_VALUES, kappa)
    got = apply(M, u, dtype)
    assert_multi_unit(M.last_launch(pmg.KERNEL_MASS))
    assert rel_err(got, oracle.mass_vmult(p, idx, jxw * kappa, cons, u)) < TOL[dtype]
    A = pmg.LaplaceOperator(mesh, p, dtype, pmg.GEOMETRY_FULL, pmg.COEFF_VALUES, kappa)
    td = tdtype(dtype)
    out = A.qp_form(torch.tensor(u, dtype=td, device="cuda"), torch.tensor(v, dtype=td, device="cuda"), -0.5)
    torch.cuda.synchronize()
    assert_multi_unit(A.last_launch(pmg.KERNEL_QP_FORM))
    G = oracle.geometry_G(ob, p, 0, kappa.reshape(-1))
    want = oracle.qp_form(p, idx, G, u, v, -0.5)
    assert rel_err(out.cpu().numpy(), want) < (TOL[dtype] if dtype == pmg.F64 else 1e-4)
