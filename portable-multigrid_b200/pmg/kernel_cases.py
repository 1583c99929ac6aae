"""Representative launches of every kernel on the path, for profilers.

    PYTHONPATH=portable-multigrid_b200 python -m pmg.kernel_cases <case> [--refine R]

Each case sets up its operators outside the NVTX range ``prof`` and runs the launches to be
profiled inside it (``ncu --nvtx --nvtx-include prof/ ...``).  The V-cycle runs as plain
launches (PMG_MG_GRAPH=0 is set here), so every kernel is visible.

  q6_kappa   the mixed-precision ph-multigrid of the Q6 variable-coefficient problem
             (3^3 coarse cells refined R times, default 4 = 48^3 cells): one FP64 CG
             iteration preconditioned by one FP32 V-cycle (operator, Chebyshev, transfer,
             conversion, residual, dot and CG-update kernels)
  dg_q3      DG-SIPG Q3 on 2^R cells per axis (default 6 = 64^3): one FP64 CG iteration with
             the FP32 DG -> CG Q3 -> Q1 -> h multigrid (cell and face kernels, DG transfer)
  adjoint_q4 Q4 on 2^R cells per axis (default 6 = 64^3): the mass matrix and the per-point
             form kernels of the adjoint gradient, FP64
"""
from __future__ import annotations

import argparse
import os

os.environ.setdefault("PMG_MG_GRAPH", "0")

import torch  # noqa: E402

import pmg  # noqa: E402


def _one_cg_iteration(h, b):
    x = h.fine64.initialize_dof_vector()
    pmg.solve_cg(h.fine64, x, b, h.mg, 1e-10, 1e-16, 1, raise_on_noconv=False)


def _range(fn):
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("prof")
    fn()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()


def q6_kappa(refine: int):
    box = pmg.Box.make(coarse=(3, 3, 3), refine=refine)
    h = pmg.Hierarchy(box, [6, 3, 2, 1], mg_dtype=pmg.F32, cheb_degree=4, geometry=pmg.GEOMETRY_AFFINE,
                      coeff_kind=pmg.COEFF_KAPPA)
    b = h.fine64.assemble_rhs(0)
    h.estimate()
    _one_cg_iteration(h, b)
    _range(lambda: _one_cg_iteration(h, b))


def dg_q3(refine: int):
    p = 3
    box = pmg.Box.make(refine=refine)
    h = pmg.Hierarchy(box, [3, 1], mg_dtype=pmg.F32, cheb_degree=5, dg=True, penalty=2.0 * (p + 1) ** 2)
    b = h.fine64.assemble_rhs(2, p + 2)
    h.estimate()
    _one_cg_iteration(h, b)
    _range(lambda: _one_cg_iteration(h, b))


def adjoint_q4(refine: int):
    box = pmg.Box.make(refine=refine)
    mesh = pmg.Mesh(box)
    op = pmg.LaplaceOperator(mesh, 4, pmg.F64, pmg.GEOMETRY_AFFINE, pmg.COEFF_VALUES)
    xq = op.quadrature_points()
    op.set_coefficient(torch.exp(0.5 * torch.sin(3.0 * xq[..., 0]) * torch.cos(2.0 * xq[..., 1])))
    M = pmg.MassOperator(mesh, 4, pmg.F64)
    u = torch.rand(M.m(), dtype=torch.float64, device="cuda")
    v = torch.rand_like(u)
    out = torch.empty_like(u)
    g = op.qp_form(u, v, -1.0)

    def run():
        M.vmult(out, u)
        op.qp_form(u, v, -1.0, out=g)

    run()
    _range(run)


CASES = {"q6_kappa": (q6_kappa, 4), "dg_q3": (dg_q3, 6), "adjoint_q4": (adjoint_q4, 6)}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--refine", type=int, default=None)
    args = ap.parse_args()
    fn, default_refine = CASES[args.case]
    fn(default_refine if args.refine is None else args.refine)
    print(f"{args.case}: done")


if __name__ == "__main__":
    main()
