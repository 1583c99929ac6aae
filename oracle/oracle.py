"""ctypes wrapper of the CPU oracle (oracle/pmg_oracle.c).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arms, never by the library.  See pmg_oracle.c for what each function
restates and how the restatement is pinned.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

INVALID = 0xFFFFFFFF


class Box(C.Structure):
    """Box mesh: coarse[0..2] coarse cells per axis, each refined `refine` times."""

    _fields_ = [
        ("coarse", C.c_int32 * 3),
        ("refine", C.c_int32),
        ("lo", C.c_double * 3),
        ("hi", C.c_double * 3),
        ("deform", C.c_int32),
        ("amp", C.c_double),
        ("dirichlet_mask", C.c_int32),
    ]

    @staticmethod
    def make(coarse=(1, 1, 1), refine=0, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), deform=0,
             amp=0.1, dirichlet_mask=0x3F):
        b = Box()
        b.coarse[:] = list(coarse)
        b.refine = refine
        b.lo[:] = list(lo)
        b.hi[:] = list(hi)
        b.deform = deform
        b.amp = amp
        b.dirichlet_mask = dirichlet_mask
        return b

    def ncells(self):
        return int(np.prod([c << self.refine for c in self.coarse]))


def doubling_box(cycle: int) -> Box:
    """The "doubling" mesh of tests/poisson_cube_bk3/program.cc:937-957 for a cycle."""
    n_refine, remainder = cycle // 3, cycle % 3
    coarse = [2 if d < remainder else 1 for d in range(3)]
    hi = [2.8 if d < remainder else 0.9 for d in range(3)]
    return Box.make(coarse=coarse, refine=n_refine, lo=(-1.0, -1.0, -1.0), hi=hi)


class SolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("n_levels", C.c_int32),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
        ("reduction_per_step", C.c_double),
        ("l2_error", C.c_double),
        ("n_dofs", C.c_int64),
        ("level_degree", C.c_int32 * 32),
        ("level_cheb_degree", C.c_int32 * 32),
        ("level_max_ev", C.c_double * 32),
        ("level_min_ev", C.c_double * 32),
        ("level_dofs", C.c_int64 * 32),
    ]


def build():
    """Compile liboracle.so from pmg_oracle.c (make, portable flags)."""
    root = os.path.dirname(_HERE)
    subprocess.run(["make", "-s", "-f", os.path.join("oracle", "Makefile"), "oracle/liboracle.so"],
                   cwd=root, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
                os.path.join(_HERE, "pmg_oracle.c")):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _p(dtype):
    return np.ctypeslib.ndpointer(dtype=dtype, flags="C_CONTIGUOUS")


def _declare(L):
    d, i64, i32, u32, u8 = np.float64, np.int64, np.int32, np.uint32, np.uint8
    BP = C.POINTER(Box)
    L.orc_gauss.argtypes = [C.c_int, _p(d), _p(d)]
    L.orc_gauss_lobatto.argtypes = [C.c_int, _p(d), _p(d)]
    L.orc_shape_tables.argtypes = [C.c_int, C.c_int, _p(d), _p(d), _p(d), _p(d)]
    L.orc_projection_matrix.argtypes = [C.c_int, C.c_int, _p(d)]
    L.orc_h_prolongation_matrix.argtypes = [C.c_int, _p(d)]
    L.orc_box_ncells.argtypes = [BP]
    L.orc_box_ncells.restype = C.c_int64
    L.orc_box_cell_coords.argtypes = [BP, _p(i32), _p(i32), _p(i32)]
    L.orc_box_dofs.argtypes = [BP, C.c_int, _p(u32), _p(u8), C.c_void_p]
    L.orc_box_dofs.restype = C.c_int64
    L.orc_apply_sentinel.argtypes = [C.c_int64, _p(u32), _p(u8), _p(u32)]
    L.orc_box_G.argtypes = [BP, C.c_int, C.c_int, C.c_void_p, _p(d)]
    L.orc_box_invjac.argtypes = [BP, C.c_int, C.c_int, _p(d), _p(d)]
    L.orc_box_quadrature.argtypes = [BP, C.c_int, C.c_int, _p(d), _p(d)]
    L.orc_vmult.argtypes = [C.c_int, C.c_int64, C.c_int64, _p(u32), _p(d), _p(u8), C.c_void_p,
                            _p(d), _p(d)]
    L.orc_vmult_invjac.argtypes = [C.c_int, C.c_int64, C.c_int64, _p(u32), _p(d), _p(d), _p(u8),
                                   _p(d), _p(d)]
    L.orc_diagonal.argtypes = [C.c_int, C.c_int64, C.c_int64, _p(u32), _p(d), _p(u8), _p(d)]
    L.orc_box_rhs.argtypes = [BP, C.c_int, C.c_int, C.c_int, _p(u32), _p(u8), C.c_int64, _p(d)]
    L.orc_box_l2_error_sine.argtypes = [BP, C.c_int, C.c_int, _p(u32), _p(d)]
    L.orc_box_l2_error_sine.restype = C.c_double
    L.orc_solve_box.argtypes = [BP, _p(i32), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_double, C.c_double, C.c_int, C.POINTER(SolveInfo), C.c_void_p]
    L.orc_solve_box_hdeg.argtypes = [BP, _p(i32), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_double, C.c_double, C.c_int, C.POINTER(SolveInfo), C.c_void_p]
    L.orc_transfer_sizes.argtypes = [BP, C.c_int, C.c_int, C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.orc_transfer_apply.argtypes = [BP, C.c_int, C.c_int, C.c_int, C.c_int, _p(d), _p(d)]
    L.orc_chebyshev_apply.argtypes = [BP, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, _p(d),
                                      _p(d), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_int)]
    L.orc_num_threads.restype = C.c_int


# ---------------------------------------------------------------------------------------
def gauss(n):
    x, w = np.zeros(n), np.zeros(n)
    lib().orc_gauss(n, x, w)
    return x, w


def gauss_lobatto(n):
    x, w = np.zeros(n), np.zeros(n)
    lib().orc_gauss_lobatto(n, x, w)
    return x, w


def shape_tables(p, nq=None):
    nq = p + 1 if nq is None else nq
    S, SD = np.zeros((p + 1) * nq), np.zeros((p + 1) * nq)
    D, W = np.zeros(nq * nq), np.zeros(nq)
    lib().orc_shape_tables(p, nq, S, SD, D, W)
    return S.reshape(p + 1, nq), SD.reshape(p + 1, nq), D.reshape(nq, nq), W


def projection_matrix(pc, pf):
    P = np.zeros((pc + 1) * (pf + 1))
    lib().orc_projection_matrix(pc, pf, P)
    return P.reshape(pc + 1, pf + 1)


def h_prolongation_matrix(p):
    P = np.zeros((p + 1) * (2 * p + 1))
    lib().orc_h_prolongation_matrix(p, P)
    return P.reshape(p + 1, 2 * p + 1)


def cell_coords(box):
    C_ = box.ncells()
    cx, cy, cz = (np.zeros(C_, np.int32) for _ in range(3))
    lib().orc_box_cell_coords(C.byref(box), cx, cy, cz)
    return cx, cy, cz


def dofs(box, p):
    """Returns (plain[C, nm^3] uint32, constrained[N] uint8, idx[C, nm^3] with sentinel)."""
    C_ = box.ncells()
    nm3 = (p + 1) ** 3
    nlat = int(np.prod([p * (c << box.refine) + 1 for c in box.coarse]))
    plain = np.zeros(C_ * nm3, np.uint32)
    constrained = np.zeros(nlat, np.uint8)
    N = lib().orc_box_dofs(C.byref(box), p, plain, constrained, None)
    constrained = constrained[:N].copy()
    idx = np.zeros_like(plain)
    lib().orc_apply_sentinel(C_ * nm3, plain, constrained, idx)
    return plain.reshape(C_, nm3), constrained, idx.reshape(C_, nm3)


def dof_lattice(box, p):
    """Node-lattice coordinates (i, j, k) of every DoF, int32 [N, 3], and the lattice itself
    [L2, L1, L0] -> DoF (x fastest)."""
    C_ = box.ncells()
    nm3 = (p + 1) ** 3
    L = [p * (c << box.refine) + 1 for c in box.coarse]
    plain = np.zeros(C_ * nm3, np.uint32)
    constrained = np.zeros(int(np.prod(L)), np.uint8)
    lat = np.zeros(int(np.prod(L)), np.uint32)
    N = lib().orc_box_dofs(C.byref(box), p, plain, constrained, lat.ctypes.data_as(C.c_void_p))
    ijk = np.zeros((N, 3), np.int32)
    t = np.arange(lat.size)
    ok = lat != INVALID
    ijk[lat[ok], 0] = t[ok] % L[0]
    ijk[lat[ok], 1] = (t[ok] // L[0]) % L[1]
    ijk[lat[ok], 2] = t[ok] // (L[0] * L[1])
    return ijk, lat.reshape(L[2], L[1], L[0])


def colors(box):
    cx, cy, cz = cell_coords(box)
    return ((cx & 1) | ((cy & 1) << 1) | ((cz & 1) << 2)).astype(np.uint8)


def geometry_G(box, p, coeff_kind=0, kappa_qp=None):
    C_ = box.ncells()
    nq3 = (p + 1) ** 3
    G = np.zeros(C_ * 6 * nq3)
    kp = None
    if kappa_qp is not None:
        kappa_qp = np.ascontiguousarray(kappa_qp, dtype=np.float64)
        kp = kappa_qp.ctypes.data_as(C.c_void_p)
    lib().orc_box_G(C.byref(box), p, coeff_kind, kp, G)
    return G.reshape(C_, 6, nq3)


def invjac(box, p, coeff_kind=0):
    C_ = box.ncells()
    nq3 = (p + 1) ** 3
    iJ = np.zeros(C_ * nq3 * 9)
    jxw = np.zeros(C_ * nq3)
    lib().orc_box_invjac(C.byref(box), p, coeff_kind, iJ, jxw)
    return iJ, jxw


def vmult(p, idx, G, constrained, src, color=None):
    C_ = idx.shape[0]
    N = constrained.shape[0]
    dst = np.zeros(N)
    cp = None
    if color is not None:
        color = np.ascontiguousarray(color, dtype=np.uint8)
        cp = color.ctypes.data_as(C.c_void_p)
    lib().orc_vmult(p, C_, N, np.ascontiguousarray(idx.reshape(-1)),
                    np.ascontiguousarray(G.reshape(-1)), constrained, cp,
                    np.ascontiguousarray(src, dtype=np.float64), dst)
    return dst


def vmult_invjac(p, idx, invJ, jxw, constrained, src):
    C_ = idx.shape[0]
    N = constrained.shape[0]
    dst = np.zeros(N)
    lib().orc_vmult_invjac(p, C_, N, np.ascontiguousarray(idx.reshape(-1)), invJ, jxw, constrained,
                           np.ascontiguousarray(src, dtype=np.float64), dst)
    return dst


def diagonal(p, idx, G, constrained):
    C_ = idx.shape[0]
    N = constrained.shape[0]
    d = np.zeros(N)
    lib().orc_diagonal(p, C_, N, np.ascontiguousarray(idx.reshape(-1)),
                       np.ascontiguousarray(G.reshape(-1)), constrained, d)
    return d


def rhs(box, p, nq, f_kind, plain, constrained):
    N = constrained.shape[0]
    b = np.zeros(N)
    lib().orc_box_rhs(C.byref(box), p, nq, f_kind, np.ascontiguousarray(plain.reshape(-1)),
                      constrained, N, b)
    return b


def l2_error_sine(box, p, nq, plain, u):
    return lib().orc_box_l2_error_sine(C.byref(box), p, nq, np.ascontiguousarray(plain.reshape(-1)),
                                       np.ascontiguousarray(u, dtype=np.float64))


def solve_box(box, pseq, cheb=5, h_times=1, rhs_kind=0, coeff_kind=0, reduce=1e-9, abs_tol=1e-16,
              maxit=100, want_x=False, h_degree=1):
    """Multigrid-preconditioned CG on a box: FE_Q(h_degree) on every refinement (h-levels),
    then the degrees of pseq (descending, ending in h_degree) on the finest mesh."""
    info = SolveInfo()
    pseq = np.ascontiguousarray(pseq, dtype=np.int32)
    x = None
    xp = None
    if want_x:
        nm = pseq[0]
        N = int(np.prod([nm * (c << box.refine) + 1 for c in box.coarse]))
        x = np.zeros(N)
        xp = x.ctypes.data_as(C.c_void_p)
    rc = lib().orc_solve_box_hdeg(C.byref(box), pseq, len(pseq), h_degree, cheb, h_times, rhs_kind,
                                  coeff_kind, reduce, abs_tol, maxit, C.byref(info), xp)
    if rc != 0:
        raise ValueError("orc_solve_box failed")
    return info, x


def transfer_sizes(fine_box, pc, pf):
    a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
    if lib().orc_transfer_sizes(C.byref(fine_box), pc, pf, C.byref(a), C.byref(b), C.byref(c)):
        raise ValueError("bad transfer")
    return a.value, b.value, c.value


def transfer_apply(fine_box, pc, pf, direction, src, dst, h_times=1):
    """direction 0: dst_fine += P src_coarse; 1: dst_coarse += P^T src_fine (in place)."""
    lib().orc_transfer_apply(C.byref(fine_box), pc, pf, h_times, direction,
                             np.ascontiguousarray(src, dtype=np.float64), dst)
    return dst


def chebyshev_apply(box, p, degree, smoothing_range, eig_its, mode, src, dst):
    mn, mx, deg = C.c_double(), C.c_double(), C.c_int()
    lib().orc_chebyshev_apply(C.byref(box), p, degree, smoothing_range, eig_its, mode,
                              np.ascontiguousarray(src, dtype=np.float64), dst, C.byref(mn),
                              C.byref(mx), C.byref(deg))
    return mn.value, mx.value, deg.value


def num_threads():
    return lib().orc_num_threads()


# ---------------------------------------------------------------------------------------
# DG-SIPG
# ---------------------------------------------------------------------------------------
def _declare_dg(L):
    d, i32 = np.float64, np.int32
    BP = C.POINTER(Box)
    L.orc_dg_vmult.argtypes = [BP, C.c_int, C.c_double, _p(d), _p(d)]
    L.orc_dg_rhs.argtypes = [BP, C.c_int, C.c_int, C.c_double, _p(d)]
    L.orc_dg_l2_error.argtypes = [BP, C.c_int, C.c_int, _p(d)]
    L.orc_dg_l2_error.restype = C.c_double
    L.orc_dg_cg_transfer.argtypes = [BP, C.c_int, C.c_int, _p(d), _p(d)]
    L.orc_dg_diagonal.argtypes = [BP, C.c_int, C.c_double, _p(d)]
    L.orc_dg_diagonal_probe.argtypes = [BP, C.c_int, C.c_double, _p(d)]
    L.orc_solve_dg.argtypes = [BP, C.c_int, _p(i32), C.c_int, C.c_int, C.c_double, C.c_double,
                               C.c_int, C.c_int, C.POINTER(SolveInfo), C.c_void_p]


def _dg_lib():
    L = lib()
    if not getattr(L, "_dg_declared", False):
        _declare_dg(L)
        L._dg_declared = True
    return L


def dg_n(box, p):
    return box.ncells() * (p + 1) ** 3


def dg_vmult(box, p, c_pen, src):
    dst = np.zeros(dg_n(box, p))
    _dg_lib().orc_dg_vmult(C.byref(box), p, c_pen, np.ascontiguousarray(src, dtype=np.float64), dst)
    return dst


def dg_rhs(box, p, nq, c_pen):
    b = np.zeros(dg_n(box, p))
    _dg_lib().orc_dg_rhs(C.byref(box), p, nq, c_pen, b)
    return b


def dg_l2_error(box, p, nq, u):
    return _dg_lib().orc_dg_l2_error(C.byref(box), p, nq, np.ascontiguousarray(u, dtype=np.float64))


def dg_cg_transfer(box, p, direction, src, dst):
    """direction 0: dst_dg += P src_cg; 1: dst_cg += P^T src_dg (in place)."""
    _dg_lib().orc_dg_cg_transfer(C.byref(box), p, direction, np.ascontiguousarray(src, dtype=np.float64), dst)
    return dst


def dg_diagonal(box, p, c_pen, probe=False):
    dgl = np.zeros(dg_n(box, p))
    fn = _dg_lib().orc_dg_diagonal_probe if probe else _dg_lib().orc_dg_diagonal
    fn(C.byref(box), p, c_pen, dgl)
    return dgl


def solve_dg(box, p, pseq, cheb=5, c_pen=None, reduce=1e-10, maxit=200, nq_rhs=None, want_x=False):
    info = SolveInfo()
    c_pen = p * (p + 1.0) if c_pen is None else c_pen
    nq_rhs = p + 2 if nq_rhs is None else nq_rhs
    x = np.zeros(dg_n(box, p)) if want_x else None
    rc = _dg_lib().orc_solve_dg(C.byref(box), p, np.ascontiguousarray(pseq, dtype=np.int32), len(pseq),
                                cheb, c_pen, reduce, maxit, nq_rhs, C.byref(info),
                                x.ctypes.data_as(C.c_void_p) if want_x else None)
    if rc != 0:
        raise ValueError("orc_solve_dg failed")
    return info, x


# ---------------------------------------------------------------------------------------
# Mass matrix, per-quadrature-point forms, coefficient fields (adjoint path)
# ---------------------------------------------------------------------------------------
def _declare_adjoint(L):
    d, u32, u8 = np.float64, np.uint32, np.uint8
    BP = C.POINTER(Box)
    L.orc_mass_vmult.argtypes = [C.c_int, C.c_int64, C.c_int64, _p(u32), _p(d), _p(u8), _p(d), _p(d)]
    L.orc_mass_diagonal.argtypes = [C.c_int, C.c_int64, C.c_int64, _p(u32), _p(d), _p(u8), _p(d)]
    L.orc_qp_form.argtypes = [C.c_int, C.c_int64, _p(u32), _p(d), _p(d), _p(d), C.c_double, _p(d)]
    L.orc_coef_interpolate.argtypes = [BP, C.c_int, _p(d), BP, C.c_int, _p(d)]


def _adj_lib():
    L = lib()
    if not getattr(L, "_adj_declared", False):
        _declare_adjoint(L)
        L._adj_declared = True
    return L


def quadrature(box, p, nq=None):
    """Gauss points xq[C, nq^3, 3] and |det J| w_q [C, nq^3] on every cell."""
    nq = p + 1 if nq is None else nq
    C_ = box.ncells()
    xq = np.zeros(C_ * nq ** 3 * 3)
    jxw = np.zeros(C_ * nq ** 3)
    lib().orc_box_quadrature(C.byref(box), p, nq, xq, jxw)
    return xq.reshape(C_, nq ** 3, 3), jxw.reshape(C_, nq ** 3)


def mass_vmult(p, idx, jxw, constrained, src):
    N = constrained.shape[0]
    dst = np.zeros(N)
    _adj_lib().orc_mass_vmult(p, idx.shape[0], N, np.ascontiguousarray(idx.reshape(-1)),
                              np.ascontiguousarray(jxw.reshape(-1), dtype=np.float64), constrained,
                              np.ascontiguousarray(src, dtype=np.float64), dst)
    return dst


def mass_diagonal(p, idx, jxw, constrained):
    N = constrained.shape[0]
    d = np.zeros(N)
    _adj_lib().orc_mass_diagonal(p, idx.shape[0], N, np.ascontiguousarray(idx.reshape(-1)),
                                 np.ascontiguousarray(jxw.reshape(-1), dtype=np.float64), constrained, d)
    return d


def qp_form(p, idx, G, u, v, alpha=1.0):
    """out[C, nq^3] = alpha * grad_ref(u)^T G grad_ref(v) at every Gauss point."""
    C_ = idx.shape[0]
    out = np.zeros(C_ * (p + 1) ** 3)
    _adj_lib().orc_qp_form(p, C_, np.ascontiguousarray(idx.reshape(-1)),
                           np.ascontiguousarray(G.reshape(-1)), np.ascontiguousarray(u, dtype=np.float64),
                           np.ascontiguousarray(v, dtype=np.float64), alpha, out)
    return out.reshape(C_, (p + 1) ** 3)


def coef_interpolate(src_box, nq_src, src, dst_box, nq_dst):
    dst = np.zeros(dst_box.ncells() * nq_dst ** 3)
    _adj_lib().orc_coef_interpolate(C.byref(src_box), nq_src,
                                    np.ascontiguousarray(src.reshape(-1), dtype=np.float64),
                                    C.byref(dst_box), nq_dst, dst)
    return dst.reshape(dst_box.ncells(), nq_dst ** 3)


def cg(apply, b, diag, tol, max_iterations=5000):
    """Jacobi-preconditioned CG from x = 0 to ||r|| <= tol ||b|| (numpy; small test cases)."""
    x = np.zeros_like(b)
    r = b.copy()
    r0 = float(np.sqrt(r @ r))
    if r0 == 0.0:
        return x
    z = r / diag
    p = z.copy()
    rz = r @ z
    for _ in range(max_iterations):
        Ap = apply(p)
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        if np.sqrt(r @ r) <= tol * r0:
            return x
        z = r / diag
        rz, rz_old = r @ z, rz
        p = z + (rz / rz_old) * p
    raise RuntimeError("CG did not converge")
