"""Parity of the DG-SIPG operator (cell + fused face kernel), its diagonal, right-hand side
with weakly imposed Dirichlet data, the DG <-> CG transfer and the DG multigrid solve with
the CPU oracle, through the C ABI.  FP64 to 1e-12 relative, FP32 to 2e-5."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
import pmg  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = {pmg.F64: 1e-12, pmg.F32: 2e-5}


def rel_err(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def obox(oracle, b):
    return oracle.Box.make(coarse=tuple(b.coarse), refine=b.refine, lo=tuple(b.lo), hi=tuple(b.hi),
                           deform=b.deform, amp=b.amp, dirichlet_mask=b.dirichlet_mask)


BOXES = {
    "cube_r2": dict(refine=2),
    "ragged_3x2x1": dict(coarse=(3, 2, 1), refine=1, hi=(3.0, 2.0, 0.5)),
    "neumann_x": dict(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0), dirichlet_mask=0x3C),
    "single_cell": dict(refine=0),
    # refined twice or more: the face kernel works on 4x4x4 tiles of cells (faces inside a
    # tile once, faces on its surface from the inside with the neighbour read from memory)
    "ragged_r2": dict(coarse=(3, 2, 1), refine=2, hi=(3.0, 2.0, 0.5)),
    "neumann_r2": dict(coarse=(2, 1, 1), refine=2, hi=(2.0, 1.0, 1.0), dirichlet_mask=0x3C),
}


def tile_form(box, p, dtype):
    """True where the face kernel can take the tile form: the box refined at least twice and
    its shared memory (a 64 x 6 int table, two face-point arrays of 240 faces, then the 64
    cells' values at a padded stride, or two more face-point arrays where those are larger
    and the face mass does not run on shuffles) within 200 KiB."""
    n = p + 1
    fp, cells = 2 * 240 * n * n, 64 * (n ** 3 + 1)
    region = cells if (32 % (n * n) == 0 or cells > fp) else fp
    size = 4 * 384 + (8 if dtype == pmg.F64 else 4) * (fp + region)
    return box.refine >= 2 and size <= 200 * 1024


@pytest.mark.parametrize("p", [1, 2, 3, 4, 6])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("boxname", list(BOXES))
def test_dg_vmult_matches_oracle(oracle, p, dtype, boxname):
    box = pmg.Box.make(**BOXES[boxname])
    ob = obox(oracle, box)
    for c_pen in (0.0, 2.0 * (p + 1) ** 2):
        op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype, c_pen)
        assert op.m() == oracle.dg_n(ob, p)
        src = np.random.default_rng(p).uniform(-1, 1, op.m())
        ref = oracle.dg_vmult(ob, p, c_pen if c_pen > 0 else p * (p + 1.0), src)
        td = torch.float64 if dtype == pmg.F64 else torch.float32
        d = op.initialize_dof_vector()
        op.vmult(d, torch.tensor(src, dtype=td, device="cuda"))
        torch.cuda.synchronize()
        assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype], c_pen


@pytest.mark.parametrize("p", [1, 2, 3, 4, 6])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("boxname", ["cube_r2", "ragged_r2", "neumann_r2"])
@pytest.mark.parametrize("fuse", ["1", "0"])
def test_dg_tile_form_matches_oracle(oracle, monkeypatch, p, dtype, boxname, fuse):
    """The tile form of the face kernel (forced with PMG_DG_FACE=2, which the library reads at
    every launch; by default it takes it only where the tiles fill the device twice) on
    meshes of 1 to 12 tiles, with Dirichlet and Neumann faces on the tile surfaces; at p = 1, 3
    the cell term runs in the same tile kernel unless PMG_DG_FUSE=0."""
    monkeypatch.setenv("PMG_DG_FACE", "2")
    monkeypatch.setenv("PMG_DG_FUSE", fuse)
    box = pmg.Box.make(**BOXES[boxname])
    ob = obox(oracle, box)
    c_pen = 2.0 * (p + 1) ** 2
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype, c_pen)
    src = np.random.default_rng(p).uniform(-1, 1, op.m())
    ref = oracle.dg_vmult(ob, p, c_pen, src)
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    s = torch.tensor(src, dtype=td, device="cuda")
    d = op.initialize_dof_vector()
    op.vmult(d, s)
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype]
    units, _ = op.last_launch(pmg.KERNEL_DG_FACES)
    n_cells = op.m() // (p + 1) ** 3
    if tile_form(box, p, dtype):
        assert units == n_cells // 64
        # with the fused kernel the cell record describes the same tile launch
        assert (op.last_launch(pmg.KERNEL_VMULT_CELL)[0] == n_cells // 64) == (fuse == "1" and p in (1, 3))
        # the tile form sums each node's faces in a fixed order: a second application, from
        # a source that is not 16-byte aligned, gives the same bits
        buf = torch.zeros(op.m() + 1, dtype=td, device="cuda")
        buf[1:] = s
        d2 = torch.empty_like(d)
        op.vmult(d2, buf[1:])
        torch.cuda.synchronize()
        assert torch.equal(d, d2)
    else:
        assert units == -(-n_cells // max(1, 384 // (6 * (p + 1) ** 2)))


@pytest.mark.parametrize("p", [1, 3, 5])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_dg_diagonal_matches_oracle(oracle, p, dtype):
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0), dirichlet_mask=0x3E)
    ob = obox(oracle, box)
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype)
    op.compute_diagonal()
    inv = op.get_matrix_diagonal_inverse()
    torch.cuda.synchronize()
    ref = oracle.dg_diagonal(ob, p, p * (p + 1.0))
    assert rel_err(1.0 / inv.double().cpu().numpy(), ref) < TOL[dtype] * 10


@pytest.mark.parametrize("p", [1, 3])
def test_dg_rhs_matches_oracle(oracle, p):
    box = pmg.Box.make(refine=2)
    ob = obox(oracle, box)
    c_pen = 2.0 * (p + 1) ** 2
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, pmg.F64, c_pen)
    b = op.assemble_rhs(2, p + 2)
    torch.cuda.synchronize()
    assert rel_err(b.cpu().numpy(), oracle.dg_rhs(ob, p, p + 2, c_pen)) < 1e-12


@pytest.mark.parametrize("p", [1, 3])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_dg_cg_transfer_matches_oracle(oracle, p, dtype):
    box = pmg.Box.make(coarse=(2, 1, 1), refine=1, hi=(2.0, 1.0, 1.0))
    ob = obox(oracle, box)
    mesh = pmg.Mesh(box)
    cg = pmg.LaplaceOperator(mesh, p, dtype)
    dg = pmg.DGLaplaceOperator(mesh, p, dtype)
    t = pmg.Transfer(cg, dg)
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    rng = np.random.default_rng(3)
    xc, xf = rng.uniform(-1, 1, cg.m()), rng.uniform(-1, 1, dg.m())
    ref = oracle.dg_cg_transfer(ob, p, 0, xc, np.zeros(dg.m()))
    d = torch.zeros(dg.m(), dtype=td, device="cuda")
    t.prolongate_and_add(d, torch.tensor(xc, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype]
    ref = oracle.dg_cg_transfer(ob, p, 1, xf, np.zeros(cg.m()))
    d = torch.zeros(cg.m(), dtype=td, device="cuda")
    t.restrict_and_add(d, torch.tensor(xf, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), ref) < TOL[dtype] * 10


@pytest.mark.parametrize("mg_dtype", [pmg.F64, pmg.F32])
def test_dg_multigrid_solve_matches_oracle(oracle, mg_dtype):
    """DG Q3 -> CG Q3 -> CG Q1 -> h-levels, penalty 2 (p+1)^2, manufactured
    u = exp(x) sin(pi y) cos(pi z) with weak Dirichlet data, FP64 CG to 1e-10."""
    p = 3
    box = pmg.Box.make(refine=2)
    ob = obox(oracle, box)
    c_pen = 2.0 * (p + 1) ** 2
    info_o, x_o = oracle.solve_dg(ob, p, [3, 1], cheb=5, c_pen=c_pen, reduce=1e-10, nq_rhs=p + 2,
                                  want_x=True)
    h = pmg.Hierarchy(box, [3, 1], mg_dtype=mg_dtype, cheb_degree=5, dg=True, penalty=c_pen)
    b = h.fine64.assemble_rhs(2, p + 2)
    x, info = h.solve(b, reduce=1e-10, max_iterations=200)
    torch.cuda.synchronize()
    assert info["converged"]
    assert abs(info["iterations"] - info_o.iterations) <= (0 if mg_dtype == pmg.F64 else 1)
    assert rel_err(x.cpu().numpy(), x_o) < 1e-7
    assert abs(oracle.dg_l2_error(ob, p, p + 2, x.cpu().numpy()) / info_o.l2_error - 1) < 1e-6


@pytest.mark.parametrize("p", [1, 3, 4])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
def test_dg_l2_error_matches_oracle(oracle, p, dtype):
    """||u_h - exp(x) sin(pi y) cos(pi z)||_L2 of a DG function on the GPU against the oracle."""
    box = pmg.Box.make(coarse=(3, 2, 1), refine=1, hi=(3.0, 2.0, 0.5))
    ob = obox(oracle, box)
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype)
    u = np.random.default_rng(3).uniform(-1, 1, op.m())
    ut = torch.tensor(u, dtype=torch.float64 if dtype == pmg.F64 else torch.float32, device="cuda")
    u_used = ut.double().cpu().numpy()
    got = op.l2_error(ut, 2, p + 2)
    want = oracle.dg_l2_error(ob, p, p + 2, u_used)
    assert abs(got - want) <= 1e-12 * want


@pytest.mark.parametrize("p,dtype", [(3, pmg.F32), (3, pmg.F64), (1, pmg.F64)])
def test_dg_vmult_with_unaligned_vectors(p, dtype):
    """The face kernel reads x-normal lines with 16-byte loads only when src is 16-byte
    aligned; a vector that starts one entry into its allocation takes the scalar loads and
    must give the same result."""
    box = pmg.Box.make(refine=2)
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype)
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    m = op.m()
    g = torch.Generator(device="cuda").manual_seed(3)
    src = torch.rand(m, generator=g, device="cuda", dtype=torch.float64).to(td)
    buf = torch.zeros(m + 1, device="cuda", dtype=td)
    buf[1:] = src
    s_off = buf[1:]
    assert s_off.data_ptr() % 16 != 0
    d0, d1 = torch.empty_like(src), torch.empty_like(src)
    op.vmult(d0, src)
    op.vmult(d1, s_off)
    torch.cuda.synchronize()
    assert torch.equal(d0, d1)


@pytest.mark.parametrize("form", ["0", "1"])
@pytest.mark.parametrize("p", [1, 3, 4])
@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("boxname", ["cube_r2", "ragged_3x2x1", "neumann_r2"])
def test_dg_face_forms_match_oracle(oracle, monkeypatch, form, p, dtype, boxname):
    """The comparison forms of the face kernel, selected at every launch: PMG_DG_FACE=0 (the
    six faces one after another) and 1 (the cell-batch kernel, also where tiles would apply)."""
    monkeypatch.setenv("PMG_DG_FACE", form)
    box = pmg.Box.make(**BOXES[boxname])
    ob = obox(oracle, box)
    c_pen = 2.0 * (p + 1) ** 2
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype, c_pen)
    src = np.random.default_rng(p).uniform(-1, 1, op.m())
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    d = op.initialize_dof_vector()
    op.vmult(d, torch.tensor(src, dtype=td, device="cuda"))
    torch.cuda.synchronize()
    assert rel_err(d.double().cpu().numpy(), oracle.dg_vmult(ob, p, c_pen, src)) < TOL[dtype]
    units, _ = op.last_launch(pmg.KERNEL_DG_FACES)
    n_cells = op.m() // (p + 1) ** 3
    batch = 128 // (p + 1) ** 2 if form == "0" else max(1, 384 // (6 * (p + 1) ** 2))
    assert units == -(-n_cells // batch)


@pytest.mark.parametrize("dtype", [pmg.F64, pmg.F32])
@pytest.mark.parametrize("p", [1, 3])
def test_dg_chebyshev_steps_in_tile_kernel(monkeypatch, dtype, p):
    """On cell tiles the Chebyshev steps of a DG smoother run inside the fused tile kernel (the
    step applied where A x is formed, A x never stored); vmult from zero and step give the
    results of the separate vmult and vector update (PMG_DG_FUSE=0)."""
    monkeypatch.setenv("PMG_DG_FACE", "2")
    box = pmg.Box.make(coarse=(2, 1, 1), refine=2, hi=(2.0, 1.0, 1.0), dirichlet_mask=0x3C)
    op = pmg.DGLaplaceOperator(pmg.Mesh(box), p, dtype, 2.0 * (p + 1) ** 2)
    op.compute_diagonal()
    td = torch.float64 if dtype == pmg.F64 else torch.float32
    src = torch.tensor(np.random.default_rng(7).uniform(-1, 1, op.m()), dtype=td, device="cuda")
    got = {}
    for fuse in ("1", "0"):
        monkeypatch.setenv("PMG_DG_FUSE", fuse)
        sm = pmg.Chebyshev(op, degree=5, smoothing_range=15.0, eig_cg_n_iterations=10)
        sm.estimate()
        d = op.initialize_dof_vector()
        sm.vmult(d, src)
        d2 = d.clone()
        sm.step(d2, src)
        torch.cuda.synchronize()
        got[fuse] = (d.double().cpu().numpy(), d2.double().cpu().numpy())
    tol = 1e-12 if dtype == pmg.F64 else 1e-5
    for a, b in zip(got["1"], got["0"]):
        assert rel_err(a, b) < tol


@pytest.mark.parametrize("mg_dtype", [pmg.F64, pmg.F32])
def test_dg_multigrid_solve_with_tiles_matches_oracle(oracle, monkeypatch, mg_dtype):
    """The DG multigrid solve of test_dg_multigrid_solve_matches_oracle with the tile forms
    forced (PMG_DG_FACE=2): the fused tile kernel applies the DG vmults and the Chebyshev
    steps of the DG level."""
    monkeypatch.setenv("PMG_DG_FACE", "2")
    p = 3
    box = pmg.Box.make(refine=2)
    ob = obox(oracle, box)
    c_pen = 2.0 * (p + 1) ** 2
    info_o, x_o = oracle.solve_dg(ob, p, [3, 1], cheb=5, c_pen=c_pen, reduce=1e-10, nq_rhs=p + 2,
                                  want_x=True)
    h = pmg.Hierarchy(box, [3, 1], mg_dtype=mg_dtype, cheb_degree=5, dg=True, penalty=c_pen)
    b = h.fine64.assemble_rhs(2, p + 2)
    x, info = h.solve(b, reduce=1e-10, max_iterations=200)
    torch.cuda.synchronize()
    assert info["converged"]
    assert abs(info["iterations"] - info_o.iterations) <= (0 if mg_dtype == pmg.F64 else 1)
    assert rel_err(x.cpu().numpy(), x_o) < 1e-7
