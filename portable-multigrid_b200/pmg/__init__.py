"""Python bindings of libpmg_b200.so over its C ABI (include/pmg/pmg.h).

The classes mirror the reference's C++ interfaces for the matrix-free multigrid path so
that code written against those reads the same here:

  LaplaceOperator  ~ Portable::LaplaceOperatorBase / LaplaceOperatorBK3
                     (vmult, Tvmult, vmult_dummy, compute_diagonal,
                      get_matrix_diagonal_inverse, m, n, el)
  Transfer         ~ Portable::MGTransferBase (prolongate_and_add, restrict_and_add)
  Chebyshev        ~ deal.II PreconditionChebyshev (vmult, step)
  VCycleMultigrid  ~ Portable::VCycleMultigridBase (vmult)
  solve_cg         ~ MultigridSolver::solve_cg

Vectors are torch CUDA tensors (float64 or float32) on the operator's device; the
library works on the tensors' memory in place, ordered on torch's current stream.
There is no CPU fallback: without the built library or a CUDA device every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
LIB_PATH = os.path.join(PKG_ROOT, "libpmg_b200.so")
HEADER_PATH = os.path.join(REPO_ROOT, "include", "pmg", "pmg.h")

F64, F32 = 0, 1
GEOMETRY_AUTO, GEOMETRY_FULL, GEOMETRY_AFFINE, GEOMETRY_INVJAC = 0, 1, 2, 3
COEFF_NONE, COEFF_KAPPA, COEFF_VALUES = 0, 1, 2
OP_LAPLACE, OP_DG_SIPG, OP_MASS = 0, 1, 2
KERNEL_VMULT_CELL, KERNEL_DG_FACES, KERNEL_MASS, KERNEL_QP_FORM = 0, 1, 2, 3
MAPS_G, MAPS_INVJAC = 0, 1
TRANSFER_POLYNOMIAL, TRANSFER_GEOMETRIC, TRANSFER_DG_CG = 0, 1, 2
INVALID = 0xFFFFFFFF
STATUS = {0: "PMG_OK", -1: "PMG_EINVAL", -2: "PMG_ENOMEM", -3: "PMG_ECUDA",
          -4: "PMG_ENONFINITE", -5: "PMG_ENOCONV", -6: "PMG_EBOUNDS", -7: "PMG_ESTATE",
          -8: "PMG_ENODEV"}


class PmgError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Box(C.Structure):
    _fields_ = [("coarse", C.c_int32 * 3), ("refine", C.c_int32), ("lo", C.c_double * 3),
                ("hi", C.c_double * 3), ("deform", C.c_int32), ("amp", C.c_double),
                ("dirichlet_mask", C.c_int32)]

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

    def with_refine(self, r):
        return Box.make(tuple(self.coarse), r, tuple(self.lo), tuple(self.hi), self.deform,
                        self.amp, self.dirichlet_mask)

    def ncells(self):
        return int(np.prod([c << self.refine for c in self.coarse]))


def doubling_box(cycle: int) -> Box:
    """The "doubling" mesh of the reference benchmark (tests/poisson_cube_bk3/program.cc:937-957)."""
    n_refine, remainder = cycle // 3, cycle % 3
    coarse = [2 if d < remainder else 1 for d in range(3)]
    hi = [2.8 if d < remainder else 0.9 for d in range(3)]
    return Box.make(coarse=coarse, refine=n_refine, lo=(-1.0, -1.0, -1.0), hi=hi)


class OperatorParams(C.Structure):
    _fields_ = [("degree", C.c_int32), ("dtype", C.c_int32), ("geometry", C.c_int32),
                ("coeff_kind", C.c_int32), ("coeff_qp", C.c_void_p), ("device", C.c_int32),
                ("kind", C.c_int32), ("penalty", C.c_double)]


class ChebyshevParams(C.Structure):
    _fields_ = [("degree", C.c_int32), ("smoothing_range", C.c_double),
                ("eig_cg_n_iterations", C.c_int32)]


class CGInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32),
                ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("reduction_per_step", C.c_double)]


class OperatorMaps(C.Structure):
    _fields_ = [("n_cells", C.c_int64), ("n_dofs", C.c_int64), ("dof_indices", C.c_void_p),
                ("constrained", C.c_void_p), ("n_constrained", C.c_int64), ("geometry", C.c_int32),
                ("G", C.c_void_p), ("inv_jacobian", C.c_void_p), ("JxW", C.c_void_p)]


class TransferMaps(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_patches", C.c_int64), ("coarse_indices", C.c_void_p),
                ("fine_indices", C.c_void_p), ("weights", C.c_void_p)]


class Peaks(C.Structure):
    _fields_ = [("copy_gbs", C.c_double), ("fp64_fma_tflops", C.c_double), ("fp32_fma_tflops", C.c_double),
                ("copy_bytes", C.c_int64), ("sm_count", C.c_int32)]


_lib = None


def build(jobs: int = 8):
    """Compile libpmg_b200.so for sm_100a (make in the package directory)."""
    subprocess.run(["make", "-s", "-j", str(jobs)], cwd=PKG_ROOT, check=True)


def header_functions():
    """Names of the functions include/pmg/pmg.h declares."""
    with open(HEADER_PATH) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pmg_[a-z0-9_]+)\s*\(", text)))


def lib():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PmgError(-8, f"{LIB_PATH} is missing: build it with pmg.build()")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    vp, i32, i64, d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    P = C.POINTER
    sig = {
        "pmg_last_error": ([C.c_char_p, C.c_size_t], C.c_size_t),
        "pmg_status_string": ([i32], C.c_char_p),
        "pmg_version": ([P(i32), P(i32)], i32),
        "pmg_mesh_create_box": ([P(Box), P(vp)], i32),
        "pmg_mesh_destroy": ([vp], i32),
        "pmg_mesh_n_cells": ([vp, P(i64)], i32),
        "pmg_mesh_cell_coordinates": ([vp, vp], i32),
        "pmg_vector_chebyshev_step": ([vp, vp, vp, vp, vp, vp, d, d, i32, i64, vp], i32),
        "pmg_operator_create": ([vp, P(OperatorParams), P(vp)], i32),
        "pmg_operator_destroy": ([vp], i32),
        "pmg_operator_create_from_maps": ([P(OperatorMaps), P(OperatorParams), P(vp)], i32),
        "pmg_transfer_create_from_maps": ([vp, vp, P(TransferMaps), P(vp)], i32),
        "pmg_operator_m": ([vp, P(i64)], i32),
        "pmg_operator_n": ([vp, P(i64)], i32),
        "pmg_operator_n_cells": ([vp, P(i64)], i32),
        "pmg_operator_degree": ([vp, P(i32), P(i32)], i32),
        "pmg_operator_vmult": ([vp, vp, vp, vp], i32),
        "pmg_operator_tvmult": ([vp, vp, vp, vp], i32),
        "pmg_operator_vmult_dummy": ([vp, vp, vp, i32, i32, vp], i32),
        "pmg_operator_vmult_cells": ([vp, vp, vp, i64, i64, i32, vp], i32),
        "pmg_operator_cells_per_group": ([vp, P(i32)], i32),
        "pmg_operator_compute_diagonal": ([vp, vp], i32),
        "pmg_operator_get_inverse_diagonal": ([vp, P(vp)], i32),
        "pmg_operator_copy_inverse_diagonal": ([vp, vp, vp], i32),
        "pmg_operator_el": ([vp, i64, i64, P(d)], i32),
        "pmg_operator_bytes_per_vmult": ([vp, P(i64)], i32),
        "pmg_operator_assemble_rhs": ([vp, i32, i32, vp, vp], i32),
        "pmg_operator_copy_dof_indices": ([vp, vp], i32),
        "pmg_operator_copy_constrained": ([vp, vp], i32),
        "pmg_operator_copy_geometry": ([vp, vp], i32),
        "pmg_operator_last_launch": ([vp, i32, P(i64), P(i64)], i32),
        "pmg_transfer_last_launch": ([vp, P(i64), P(i64)], i32),
        "pmg_operator_set_coefficient": ([vp, vp, i32, vp], i32),
        "pmg_operator_interpolate_coefficient": ([vp, vp, vp], i32),
        "pmg_operator_quadrature_points": ([vp, vp, vp], i32),
        "pmg_operator_l2_error": ([vp, vp, i32, i32, P(d), vp], i32),
        "pmg_operator_dof_coordinates": ([vp, vp, vp], i32),
        "pmg_operator_qp_form": ([vp, vp, vp, d, vp, vp], i32),
        "pmg_mg_set_coefficient": ([vp, vp, vp, i32, vp], i32),
        "pmg_adjoint_gradient": ([vp, vp, vp, vp, vp, vp, vp, P(d), d, d, i32, P(CGInfo), vp], i32),
        "pmg_transfer_create": ([vp, vp, P(vp)], i32),
        "pmg_transfer_destroy": ([vp], i32),
        "pmg_transfer_prolongate_and_add": ([vp, vp, vp, vp], i32),
        "pmg_transfer_restrict_and_add": ([vp, vp, vp, vp], i32),
        "pmg_chebyshev_create": ([vp, P(ChebyshevParams), P(vp)], i32),
        "pmg_chebyshev_destroy": ([vp], i32),
        "pmg_chebyshev_estimate": ([vp, vp], i32),
        "pmg_chebyshev_vmult": ([vp, vp, vp, vp], i32),
        "pmg_chebyshev_step": ([vp, vp, vp, vp], i32),
        "pmg_chebyshev_info": ([vp, P(d), P(d), P(i32), P(i32)], i32),
        "pmg_mg_create": ([i32, P(vp), P(vp), P(vp), P(vp)], i32),
        "pmg_mg_destroy": ([vp], i32),
        "pmg_mg_vmult": ([vp, vp, vp, i32, vp], i32),
        "pmg_cg_solve": ([vp, vp, vp, vp, d, d, i32, P(CGInfo), vp], i32),
        "pmg_vector_dot": ([vp, vp, i32, i64, P(d), vp], i32),
        "pmg_vector_copy": ([vp, i32, vp, i32, i64, vp], i32),
        "pmg_vector_axpy": ([vp, vp, d, i32, i64, vp], i32),
        "pmg_vector_xpay": ([vp, vp, d, i32, i64, vp], i32),
        "pmg_vector_pointwise_mult": ([vp, vp, vp, i32, i64, vp], i32),
        "pmg_operator_dof_lattice": ([vp, vp], i32),
        "pmg_operator_set_tensor_cores": ([vp, i32], i32),
        "pmg_profile_enable": ([i32], i32),
        "pmg_profile_reset": ([], i32),
        "pmg_profile_query": ([C.c_char_p, P(d), P(i64)], i32),
        "pmg_measure_peaks": ([i32, i64, P(Peaks)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res


def last_error() -> str:
    buf = C.create_string_buffer(2048)
    lib().pmg_last_error(buf, 2048)
    return buf.value.decode(errors="replace")


def check(status):
    if status != 0:
        raise PmgError(status, last_error())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _dt(t):
    import torch
    return F64 if t.dtype == torch.float64 else F32


def vector_dot(a, b):
    """sum(a*b) of two device vectors of the same dtype, accumulated in FP64."""
    r = C.c_double()
    check(lib().pmg_vector_dot(_ptr(a), _ptr(b), _dt(a), a.numel(), C.byref(r), _stream()))
    return r.value


def vector_copy(dst, src):
    """dst = src with precision conversion (copy_locally_owned_data_from)."""
    check(lib().pmg_vector_copy(_ptr(dst), _dt(dst), _ptr(src), _dt(src), src.numel(), _stream()))


def vector_axpy(y, x, alpha):
    """y += alpha x (device vectors of one dtype)."""
    check(lib().pmg_vector_axpy(_ptr(y), _ptr(x), float(alpha), _dt(y), y.numel(), _stream()))


def vector_xpay(y, x, alpha):
    """y = x + alpha y."""
    check(lib().pmg_vector_xpay(_ptr(y), _ptr(x), float(alpha), _dt(y), y.numel(), _stream()))


def vector_pointwise_mult(z, d, r):
    """z = d .* r."""
    check(lib().pmg_vector_pointwise_mult(_ptr(z), _ptr(d), _ptr(r), _dt(z), z.numel(), _stream()))


def vector_chebyshev_step(out, cur, prev, src, Ax, inv_diag, f1, f2):
    """out = cur + f1 (cur - prev) + f2 inv_diag .* (src - Ax); prev None means zero."""
    check(lib().pmg_vector_chebyshev_step(_ptr(out), _ptr(cur), None if prev is None else _ptr(prev), _ptr(src),
                                          _ptr(Ax), _ptr(inv_diag), float(f1), float(f2), _dt(out), out.numel(),
                                          _stream()))


def profile_enable(on=True):
    check(lib().pmg_profile_enable(int(on)))


def profile_reset():
    check(lib().pmg_profile_reset())


def profile_query(kernel):
    """(total device milliseconds, launches) of a kernel label since the last reset."""
    ms, n = C.c_double(), C.c_int64()
    check(lib().pmg_profile_query(kernel.encode(), C.byref(ms), C.byref(n)))
    return ms.value, n.value


def measure_peaks(device: int = 0, copy_bytes: int = 1 << 30):
    """Same-run peaks on `device`: STREAM-style copy GB/s (read + write bytes) over two buffers
    of `copy_bytes`, and FP64 / FP32 FMA TFLOP/s (pmg_measure_peaks)."""
    p = Peaks()
    check(lib().pmg_measure_peaks(device, copy_bytes, C.byref(p)))
    return {"copy_gbs": p.copy_gbs, "fp64_fma_tflops": p.fp64_fma_tflops,
            "fp32_fma_tflops": p.fp32_fma_tflops, "copy_bytes": p.copy_bytes, "sm_count": p.sm_count}


class Mesh:
    def __init__(self, box: Box):
        self.box = box
        self.h = C.c_void_p()
        check(lib().pmg_mesh_create_box(C.byref(box), C.byref(self.h)))

    def n_cells(self):
        n = C.c_int64()
        check(lib().pmg_mesh_n_cells(self.h, C.byref(n)))
        return n.value

    def cell_coordinates(self):
        """Integer cell coordinates (x, y, z) in cell order, int32 [n_cells, 3] (host)."""
        out = np.zeros((self.n_cells(), 3), dtype=np.int32)
        check(lib().pmg_mesh_cell_coordinates(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pmg_mesh_destroy(self.h)
            self.h = None


class LaplaceOperator:
    """Continuous FE_Q(degree) Laplace operator on a box mesh (LaplaceOperatorBK3)."""

    def __init__(self, mesh: Mesh, degree: int, dtype: int = F64, geometry: int = GEOMETRY_AUTO,
                 coeff_kind: int = COEFF_NONE, coeff_qp=None, device: int = 0,
                 kind: int = OP_LAPLACE, penalty: float = 0.0):
        self.mesh = mesh
        self.degree = degree
        self.dtype = dtype
        self.device = device
        self.kind = kind
        self._coeff = None
        prm = OperatorParams(degree, dtype, geometry, coeff_kind, None, device, kind, penalty)
        if coeff_qp is not None:
            self._coeff = np.ascontiguousarray(coeff_qp, dtype=np.float64)
            prm.coeff_qp = self._coeff.ctypes.data_as(C.c_void_p)
        self.h = C.c_void_p()
        check(lib().pmg_operator_create(mesh.h, C.byref(prm), C.byref(self.h)))

    @classmethod
    def from_maps(cls, n_dofs, dof_indices, constrained, degree, dtype=F64, G=None, inv_jacobian=None,
                  JxW=None, device=0):
        """An operator on the caller's own discretisation (pmg_operator_create_from_maps):
        dof_indices [C, (degree+1)^3] uint32 with 0xFFFFFFFF on constrained DoFs, the list of
        constrained DoFs, and either G [C, 6, nq^3] or inv_jacobian [C, nq^3, 3, 3] with
        JxW [C, nq^3]."""
        self = cls.__new__(cls)
        self.mesh, self.degree, self.dtype, self.device, self.kind, self._coeff = None, degree, dtype, device, OP_LAPLACE, None
        idx = np.ascontiguousarray(dof_indices, dtype=np.uint32)
        cons = np.ascontiguousarray(constrained, dtype=np.uint32).reshape(-1)
        nm3 = (degree + 1) ** 3
        n_cells = idx.size // nm3
        m = OperatorMaps(n_cells, int(n_dofs), idx.ctypes.data_as(C.c_void_p), cons.ctypes.data_as(C.c_void_p),
                         cons.size, MAPS_G if G is not None else MAPS_INVJAC, None, None, None)
        keep = [idx, cons]
        if G is not None:
            g = np.ascontiguousarray(G, dtype=np.float64)
            keep.append(g)
            m.G = g.ctypes.data_as(C.c_void_p)
        else:
            ij = np.ascontiguousarray(inv_jacobian, dtype=np.float64)
            jw = np.ascontiguousarray(JxW, dtype=np.float64)
            keep += [ij, jw]
            m.inv_jacobian = ij.ctypes.data_as(C.c_void_p)
            m.JxW = jw.ctypes.data_as(C.c_void_p)
        prm = OperatorParams(degree, dtype, GEOMETRY_AUTO, COEFF_NONE, None, device, OP_LAPLACE, 0.0)
        self.h = C.c_void_p()
        check(lib().pmg_operator_create_from_maps(C.byref(m), C.byref(prm), C.byref(self.h)))
        return self

    @property
    def torch_dtype(self):
        import torch
        return torch.float64 if self.dtype == F64 else torch.float32

    def m(self):
        n = C.c_int64()
        check(lib().pmg_operator_m(self.h, C.byref(n)))
        return n.value

    n = m

    def n_cells(self):
        n = C.c_int64()
        check(lib().pmg_operator_n_cells(self.h, C.byref(n)))
        return n.value

    def initialize_dof_vector(self):
        import torch
        return torch.zeros(self.m(), dtype=self.torch_dtype, device=f"cuda:{self.device}")

    def vmult(self, dst, src):
        check(lib().pmg_operator_vmult(self.h, _ptr(dst), _ptr(src), _stream()))

    def Tvmult(self, dst, src):
        check(lib().pmg_operator_tvmult(self.h, _ptr(dst), _ptr(src), _stream()))

    def vmult_dummy(self, dst, src, ghost_exchange_on=True, computation_on=True):
        check(lib().pmg_operator_vmult_dummy(self.h, _ptr(dst), _ptr(src), int(ghost_exchange_on),
                                             int(computation_on), _stream()))

    def vmult_cells(self, dst, src, cell_begin, cell_end, init):
        """dst += A_K src over the cells [cell_begin, cell_end) of the operator's cell order;
        init first sets dst as vmult does (pmg_operator_vmult_cells)."""
        check(lib().pmg_operator_vmult_cells(self.h, _ptr(dst), _ptr(src), int(cell_begin), int(cell_end),
                                             int(bool(init)), _stream()))

    def cells_per_group(self):
        v = C.c_int32()
        check(lib().pmg_operator_cells_per_group(self.h, C.byref(v)))
        return v.value

    def compute_diagonal(self):
        check(lib().pmg_operator_compute_diagonal(self.h, _stream()))

    def get_matrix_diagonal_inverse(self):
        """Returns a torch view of the operator-owned inverse diagonal."""
        import torch
        p = C.c_void_p()
        check(lib().pmg_operator_get_inverse_diagonal(self.h, C.byref(p)))
        n = self.m()
        out = torch.empty(n, dtype=self.torch_dtype, device=f"cuda:{self.device}")
        # a copy, so the tensor does not alias library memory
        check(lib().pmg_operator_copy_inverse_diagonal(self.h, _ptr(out), _stream()))
        return out

    def el(self, row, col):
        v = C.c_double()
        check(lib().pmg_operator_el(self.h, row, col, C.byref(v)))
        return v.value

    def bytes_per_vmult(self):
        b = C.c_int64()
        check(lib().pmg_operator_bytes_per_vmult(self.h, C.byref(b)))
        return b.value

    def assemble_rhs(self, f_kind=0, nq=0):
        b = self.initialize_dof_vector()
        check(lib().pmg_operator_assemble_rhs(self.h, f_kind, nq, _ptr(b), _stream()))
        return b

    def dof_indices(self):
        nm3 = (self.degree + 1) ** 3
        out = np.zeros(self.n_cells() * nm3, dtype=np.uint32)
        check(lib().pmg_operator_copy_dof_indices(self.h, out.ctypes.data_as(C.c_void_p)))
        return out.reshape(-1, nm3)

    def set_tensor_cores(self, mode):
        """Cell kernel of an FP32 affine operator: 0 CUDA cores, 1 TF32 mma, 3 three TF32 products."""
        check(lib().pmg_operator_set_tensor_cores(self.h, int(mode)))

    def dof_lattice(self):
        """Node-lattice coordinates (i, j, k) of every DoF, int32 [m, 3] (host)."""
        out = np.zeros((self.m(), 3), dtype=np.int32)
        check(lib().pmg_operator_dof_lattice(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def constrained(self):
        out = np.zeros(self.m(), dtype=np.uint8)
        check(lib().pmg_operator_copy_constrained(self.h, out.ctypes.data_as(C.c_void_p)))
        return out

    def geometry(self):
        nq3 = (self.degree + 1) ** 3
        out = np.zeros(self.n_cells() * 6 * nq3)
        check(lib().pmg_operator_copy_geometry(self.h, out.ctypes.data_as(C.c_void_p)))
        return out.reshape(-1, 6, nq3)

    def last_launch(self, kernel=KERNEL_VMULT_CELL):
        """(work units, warps or blocks) of the last launch of one of the operator's kernels."""
        u, p = C.c_int64(), C.c_int64()
        check(lib().pmg_operator_last_launch(self.h, kernel, C.byref(u), C.byref(p)))
        return u.value, p.value

    # -- coefficient fields and per-point forms (adjoint path) --------------------------
    def set_coefficient(self, values):
        """New PMG_COEFF_VALUES values [C, nq^3]: a float64 CUDA tensor or a host array."""
        if hasattr(values, "is_cuda") and values.is_cuda:
            v = values.contiguous()
            check(lib().pmg_operator_set_coefficient(self.h, _ptr(v), 1, _stream()))
        else:
            v = np.ascontiguousarray(values, dtype=np.float64)
            check(lib().pmg_operator_set_coefficient(self.h, v.ctypes.data_as(C.c_void_p), 0, _stream()))

    def interpolate_coefficient(self, src: "LaplaceOperator"):
        """This operator's coefficient := src's coefficient field at this operator's points."""
        check(lib().pmg_operator_interpolate_coefficient(self.h, src.h, _stream()))

    def l2_error(self, u, exact_kind, nq=0):
        """||u_h - u||_L2 against the manufactured solution exact_kind (1: sine, 2: exp-sine-cosine)."""
        e = C.c_double()
        check(lib().pmg_operator_l2_error(self.h, _ptr(u), exact_kind, nq, C.byref(e), _stream()))
        return e.value

    def dof_coordinates(self):
        """Support point of every DoF, float64 CUDA tensor [m, 3]."""
        import torch
        xyz = torch.empty((self.m(), 3), dtype=torch.float64, device=f"cuda:{self.device}")
        check(lib().pmg_operator_dof_coordinates(self.h, _ptr(xyz), _stream()))
        return xyz

    def quadrature_points(self):
        """Gauss points of every cell, float64 CUDA tensor [C, nq^3, 3]."""
        import torch
        nq3 = (self.degree + 1) ** 3
        xq = torch.empty(self.n_cells(), nq3, 3, dtype=torch.float64, device=f"cuda:{self.device}")
        check(lib().pmg_operator_quadrature_points(self.h, _ptr(xq), _stream()))
        return xq

    def qp_form(self, u, v, alpha=1.0, out=None):
        """alpha * grad u^T (coefficient) G grad v at every Gauss point, float64 [C, nq^3]."""
        import torch
        nq3 = (self.degree + 1) ** 3
        if out is None:
            out = torch.empty(self.n_cells(), nq3, dtype=torch.float64, device=f"cuda:{self.device}")
        check(lib().pmg_operator_qp_form(self.h, _ptr(u), _ptr(v), alpha, _ptr(out), _stream()))
        return out

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pmg_operator_destroy(self.h)
            self.h = None


class Transfer:
    """PolynomialTransfer / GeometricTransfer between two level operators."""

    def __init__(self, coarse: LaplaceOperator, fine: LaplaceOperator):
        self.coarse, self.fine = coarse, fine
        self.h = C.c_void_p()
        check(lib().pmg_transfer_create(coarse.h, fine.h, C.byref(self.h)))

    @classmethod
    def from_maps(cls, coarse: "LaplaceOperator", fine: "LaplaceOperator", kind, coarse_indices, fine_indices,
                  weights=None):
        """A transfer from the caller's patch maps (pmg_transfer_create_from_maps)."""
        self = cls.__new__(cls)
        self.coarse, self.fine = coarse, fine
        ci = np.ascontiguousarray(coarse_indices, dtype=np.uint32)
        fi = np.ascontiguousarray(fine_indices, dtype=np.uint32)
        nc3 = (coarse.degree + 1) ** 3
        m = TransferMaps(kind, ci.size // nc3, ci.ctypes.data_as(C.c_void_p), fi.ctypes.data_as(C.c_void_p), None)
        w = None
        if weights is not None:
            w = np.ascontiguousarray(weights, dtype=np.float64)
            m.weights = w.ctypes.data_as(C.c_void_p)
        self.h = C.c_void_p()
        check(lib().pmg_transfer_create_from_maps(coarse.h, fine.h, C.byref(m), C.byref(self.h)))
        return self

    def prolongate_and_add(self, dst_fine, src_coarse):
        check(lib().pmg_transfer_prolongate_and_add(self.h, _ptr(dst_fine), _ptr(src_coarse), _stream()))

    def restrict_and_add(self, dst_coarse, src_fine):
        check(lib().pmg_transfer_restrict_and_add(self.h, _ptr(dst_coarse), _ptr(src_fine), _stream()))

    def last_launch(self):
        """(patches, warps) of the last launch."""
        u, p = C.c_int64(), C.c_int64()
        check(lib().pmg_transfer_last_launch(self.h, C.byref(u), C.byref(p)))
        return u.value, p.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pmg_transfer_destroy(self.h)
            self.h = None


class Chebyshev:
    """PreconditionChebyshev with the operator's inverse diagonal (degree <= 0: automatic)."""

    def __init__(self, op: LaplaceOperator, degree=5, smoothing_range=15.0, eig_cg_n_iterations=10):
        self.op = op
        prm = ChebyshevParams(degree, smoothing_range, eig_cg_n_iterations)
        self.h = C.c_void_p()
        check(lib().pmg_chebyshev_create(op.h, C.byref(prm), C.byref(self.h)))

    def estimate(self):
        check(lib().pmg_chebyshev_estimate(self.h, _stream()))

    def vmult(self, dst, src):
        check(lib().pmg_chebyshev_vmult(self.h, _ptr(dst), _ptr(src), _stream()))

    def step(self, dst, src):
        check(lib().pmg_chebyshev_step(self.h, _ptr(dst), _ptr(src), _stream()))

    def info(self):
        mn, mx, deg, its = C.c_double(), C.c_double(), C.c_int32(), C.c_int32()
        check(lib().pmg_chebyshev_info(self.h, C.byref(mn), C.byref(mx), C.byref(deg), C.byref(its)))
        return {"min_eigenvalue": mn.value, "max_eigenvalue": mx.value, "degree": deg.value,
                "cg_iterations": its.value}

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pmg_chebyshev_destroy(self.h)
            self.h = None


class VCycleMultigrid:
    """V-cycle over levels[0] (coarsest) .. levels[-1] (finest)."""

    def __init__(self, levels, transfers, smoothers):
        self.levels, self.transfers, self.smoothers = levels, transfers, smoothers
        n = len(levels)
        lv = (C.c_void_p * n)(*[o.h for o in levels])
        tr = (C.c_void_p * n)(*([None] + [t.h for t in transfers[1:]]))
        sm = (C.c_void_p * n)(*[s.h for s in smoothers])
        self.h = C.c_void_p()
        check(lib().pmg_mg_create(n, lv, tr, sm, C.byref(self.h)))

    def vmult(self, dst, src):
        import torch
        vd = F64 if src.dtype == torch.float64 else F32
        check(lib().pmg_mg_vmult(self.h, _ptr(dst), _ptr(src), vd, _stream()))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.pmg_mg_destroy(self.h)
            self.h = None


def MassOperator(mesh: Mesh, degree: int, dtype: int = F64, geometry: int = GEOMETRY_AUTO,
                 coeff_kind: int = COEFF_NONE, coeff_qp=None, device: int = 0):
    """FE_Q(degree) mass matrix (phi_i, coefficient phi_j), identity rows on constrained DoFs."""
    return LaplaceOperator(mesh, degree, dtype, geometry, coeff_kind, coeff_qp, device, OP_MASS)


def DGLaplaceOperator(mesh: Mesh, degree: int, dtype: int = F64, penalty: float = 0.0, device: int = 0):
    """FE_DGQ(degree) symmetric interior penalty operator (LaplaceOperatorDG); penalty <= 0
    selects the reference's p(p+1)."""
    return LaplaceOperator(mesh, degree, dtype, GEOMETRY_AFFINE, COEFF_NONE, None, device,
                           OP_DG_SIPG, penalty)


def solve_cg(A: LaplaceOperator, x, b, precond: VCycleMultigrid | None = None, reduce=1e-9,
             abs_tol=1e-16, max_iterations=100, raise_on_noconv=True):
    info = CGInfo()
    st = lib().pmg_cg_solve(A.h, precond.h if precond is not None else None, _ptr(x), _ptr(b),
                            reduce, abs_tol, max_iterations, C.byref(info), _stream())
    if st != 0 and not (st == -5 and not raise_on_noconv):
        raise PmgError(st, last_error())
    return {"iterations": info.iterations, "converged": bool(info.converged),
            "initial_residual": info.initial_residual, "final_residual": info.final_residual,
            "reduction_per_step": info.reduction_per_step}


class Hierarchy:
    """The multigrid hierarchies of the reference's drivers: FE_Q(h_degree) on every
    refinement of the box (h-levels), then the degrees of `pseq` (descending, ending in
    h_degree) on the finest mesh.  h_degree = 1 is the ph-multigrid of LaplaceProblem
    (tests/poisson_cube_bk3/program.cc:263-515); pseq = [p] with h_degree = p is the plain
    geometric multigrid of source/geometric_multigrid/program.cc:245-249
    (GeometricTransfer<dim, fe_degree> at one degree on every level).  Chebyshev(cheb_degree,
    range 15, 10 eigenvalue iterations) on levels > 0 and Chebyshev-to-1e-3 on level 0.  With
    dg=True an FE_DGQ(pseq[0]) SIPG level sits on top, connected by the DG <-> CG transfer.
    The finest-level FP64 operator `fine64` is the CG matrix."""

    def __init__(self, box: Box, pseq, mg_dtype=F32, cheb_degree=5, geometry=GEOMETRY_AUTO,
                 coeff_kind=COEFF_NONE, coeff_qp=None, device=0, smoothing_range=15.0,
                 eig_iterations=10, coarse_dtype=None, dg=False, penalty=0.0, h_degree=1, tensor_cores=0):
        if pseq[-1] != h_degree or list(pseq) != sorted(pseq, reverse=True):
            raise ValueError("pseq must be descending and end in h_degree")
        self.box = box
        coarse_dtype = mg_dtype if coarse_dtype is None else coarse_dtype
        self.meshes = [Mesh(box.with_refine(r)) for r in range(box.refine + 1)]
        self.levels, self.transfers, self.smoothers = [], [None], []
        n_h = box.refine + 1
        degrees = [h_degree] * n_h + list(reversed(pseq))[1:]
        for l, p in enumerate(degrees):
            mesh = self.meshes[min(l, n_h - 1)]
            dt = coarse_dtype if l == 0 else mg_dtype
            finest = l == len(degrees) - 1 and not dg
            self.levels.append(LaplaceOperator(mesh, p, dt, geometry, coeff_kind,
                                               coeff_qp if finest else None, device))
        if coeff_kind == COEFF_VALUES:
            # coarser levels carry the finest level's field, interpolated level by level
            for l in range(len(self.levels) - 2, -1, -1):
                self.levels[l].interpolate_coefficient(self.levels[l + 1])
        if tensor_cores:
            # the FP32 affine levels apply their cells on the tensor cores
            for op in self.levels:
                if op.dtype == F32 and geometry != GEOMETRY_FULL and not box.deform:
                    op.set_tensor_cores(tensor_cores)
        if dg:
            self.levels.append(DGLaplaceOperator(self.meshes[-1], pseq[0], mg_dtype, penalty, device))
        for l in range(1, len(self.levels)):
            if self.levels[l].dtype != self.levels[l - 1].dtype:
                raise ValueError("all multigrid levels must share one dtype")
            self.transfers.append(Transfer(self.levels[l - 1], self.levels[l]))
        for l, op in enumerate(self.levels):
            if l == 0:
                self.smoothers.append(Chebyshev(op, 0, 1e-3, op.m()))
            else:
                self.smoothers.append(Chebyshev(op, cheb_degree, smoothing_range, eig_iterations))
        if dg:
            self.fine64 = DGLaplaceOperator(self.meshes[-1], pseq[0], F64, penalty, device)
        else:
            self.fine64 = LaplaceOperator(self.meshes[-1], pseq[0], F64, geometry, coeff_kind,
                                          coeff_qp, device)
        self.mg = VCycleMultigrid(self.levels, self.transfers, self.smoothers)
        self._fine_args = (pseq[0], geometry, coeff_kind, coeff_qp, device, dg)
        self._lift_op = None

    def set_coefficient(self, values):
        """New coefficient values [C, nq^3] (float64, CUDA tensor or host array) for the CG
        matrix and every level (interpolated downwards); diagonals and smoother estimates are
        recomputed."""
        if hasattr(values, "is_cuda") and values.is_cuda:
            v = values.contiguous()
            check(lib().pmg_mg_set_coefficient(self.mg.h, self.fine64.h, _ptr(v), 1, _stream()))
        else:
            v = np.ascontiguousarray(values, dtype=np.float64)
            check(lib().pmg_mg_set_coefficient(self.mg.h, self.fine64.h, v.ctypes.data_as(C.c_void_p), 0,
                                               _stream()))

    def estimate(self):
        for s in self.smoothers:
            s.estimate()

    def solve(self, b, x=None, reduce=1e-9, abs_tol=1e-16, max_iterations=100):
        if x is None:
            x = self.fine64.initialize_dof_vector()
        info = solve_cg(self.fine64, x, b, self.mg, reduce, abs_tol, max_iterations)
        return x, info

    def solve_dirichlet(self, b, g, reduce=1e-9, abs_tol=1e-16, max_iterations=100):
        """Solve with inhomogeneous Dirichlet data by lifting (the reference imposes
        homogeneous data only).  g maps the DoF support points (float64 CUDA tensor [m, 3]) to
        the boundary values; b is the right-hand side of pmg_operator_assemble_rhs (zero on
        the Dirichlet rows).  u_D = g at the Dirichlet DoFs and 0 elsewhere; b0 = b - A0 u_D on
        the free rows, with A0 the same operator on the same mesh without Dirichlet DoFs (the
        numbering does not depend on them); u = u0 + u_D with A u0 = b0.  Returns (u, info)."""
        import torch
        degree, geometry, coeff_kind, coeff_qp, device, dg = self._fine_args
        if dg:
            raise ValueError("DG operators take Dirichlet data weakly (pmg_operator_assemble_rhs)")
        A = self.fine64
        if self._lift_op is None:
            b0x = self.box
            free_box = Box.make(tuple(b0x.coarse), b0x.refine, tuple(b0x.lo), tuple(b0x.hi), b0x.deform,
                                b0x.amp, 0)
            self._lift_mesh = Mesh(free_box)
            self._lift_op = LaplaceOperator(self._lift_mesh, degree, F64, geometry, coeff_kind, coeff_qp, device)
            self._lift_cons = torch.as_tensor(A.constrained().astype(bool), device=f"cuda:{device}")
        cons = self._lift_cons
        xyz = A.dof_coordinates()
        u_d = torch.where(cons, g(xyz).to(torch.float64), torch.zeros((), dtype=torch.float64, device=xyz.device))
        r = torch.empty_like(u_d)
        self._lift_op.vmult(r, u_d)
        b0 = torch.where(cons, torch.zeros((), dtype=torch.float64, device=xyz.device), b - r)
        u0, info = self.solve(b0, reduce=reduce, abs_tol=abs_tol, max_iterations=max_iterations)
        return u0 + u_d, info


def adjoint_gradient(A: LaplaceOperator, M: LaplaceOperator, u, u_d, precond: VCycleMultigrid | None = None,
                     reduce=1e-13, abs_tol=1e-300, max_iterations=200, lam=None, g=None):
    """J = 1/2 (u-u_d)^T M (u-u_d), the adjoint solve A lambda = M (u - u_d) and
    g[c, q] = dJ/dm_q = -exp(m_q) grad lambda^T G grad u.  Returns (J, g, lambda, cg info)."""
    import torch
    nq3 = (A.degree + 1) ** 3
    if lam is None:
        lam = A.initialize_dof_vector()
    if g is None:
        g = torch.empty(A.n_cells(), nq3, dtype=torch.float64, device=f"cuda:{A.device}")
    J = C.c_double()
    info = CGInfo()
    check(lib().pmg_adjoint_gradient(A.h, M.h, precond.h if precond is not None else None, _ptr(u), _ptr(u_d),
                                     _ptr(lam), _ptr(g), C.byref(J), reduce, abs_tol, max_iterations,
                                     C.byref(info), _stream()))
    return J.value, g, lam, {"iterations": info.iterations, "converged": bool(info.converged),
                             "initial_residual": info.initial_residual,
                             "final_residual": info.final_residual}
