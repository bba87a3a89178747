"""Host-side mirror of the reference's LAFEM containers and its Arch op-level seam.

Containers (host, numpy): ``SparseMatrixCSR`` (kernel/lafem/sparse_matrix_csr.hpp:280-302),
``DenseVector`` (kernel/lafem/dense_vector.hpp:58), ``UnitFilter`` (kernel/lafem/unit_filter.hpp:30)
and ``Transfer`` (kernel/lafem/transfer.hpp).  They carry the data the solver seam uploads.

``arch`` functions take CUDA tensors (torch, used only as device memory) and call the library's
op-level entry points, the counterparts of ``LAFEM::Arch::*`` (kernel/lafem/arch/*.hpp).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


class DenseVector:
    """DenseVector<double, Index>: a contiguous FP64 array."""

    def __init__(self, size_or_array):
        if isinstance(size_or_array, (int, np.integer)):
            self.elements = np.zeros(int(size_or_array))
        else:
            self.elements = np.ascontiguousarray(size_or_array, dtype=np.float64)

    def size(self):
        return self.elements.size

    def format(self, value=0.0):
        self.elements[:] = value

    def copy(self, other):
        self.elements[:] = other.elements

    def clone(self):
        return DenseVector(self.elements.copy())

    def norm2(self):
        return float(np.sqrt(np.dot(self.elements, self.elements)))

    # DenseVector::read_from / write_out (kernel/lafem/dense_vector.hpp:600-720); mode "dv"/"binary",
    # "mtx" or "exp" (featb200.fileio)
    @staticmethod
    def read_from(mode, filename):
        from . import fileio
        return DenseVector(fileio.read_dv(filename, mode))

    def write_out(self, mode, filename):
        from . import fileio
        fileio.write_dv(filename, self.elements, mode)


class SparseMatrixCSR:
    """SparseMatrixCSR<double, Index>: row_ptr[rows+1], col_ind[nnz] (u64), val[nnz] (f64)."""

    def __init__(self, row_ptr, col_ind, val, shape):
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.uint64)
        self.col_ind = np.ascontiguousarray(col_ind, dtype=np.uint64)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self.shape = (int(shape[0]), int(shape[1]))
        if self.row_ptr.size != self.shape[0] + 1 or self.col_ind.size != self.val.size:
            raise ValueError("inconsistent CSR arrays")

    @staticmethod
    def from_scipy(m):
        m = m.tocsr()
        m.sort_indices()
        return SparseMatrixCSR(m.indptr, m.indices, m.data, m.shape)

    def rows(self):
        return self.shape[0]

    def columns(self):
        return self.shape[1]

    def used_elements(self):
        return int(self.val.size)

    def create_vector_r(self):
        return DenseVector(self.shape[0])

    def create_vector_l(self):
        return DenseVector(self.shape[1])

    def transpose(self):
        import scipy.sparse as sp
        t = sp.csr_matrix((self.val, self.col_ind.astype(np.int64), self.row_ptr.astype(np.int64)),
                          shape=self.shape).T.tocsr()
        t.sort_indices()
        return SparseMatrixCSR(t.indptr, t.indices, t.data, t.shape)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col_ind.astype(np.int64), self.row_ptr.astype(np.int64)),
                             shape=self.shape)

    # SparseMatrixCSR::read_from / write_out (kernel/lafem/sparse_matrix_csr.hpp:880-1125); mode
    # "csr"/"binary" or "mtx" (featb200.fileio)
    @staticmethod
    def read_from(mode, filename):
        from . import fileio
        rows, cols, rp, ci, val = fileio.read_csr(filename, mode)
        return SparseMatrixCSR(rp, ci, val, (rows, cols))

    def write_out(self, mode, filename):
        from . import fileio
        fileio.write_csr(filename, self.shape[0], self.shape[1], self.row_ptr, self.col_ind, self.val, mode)

    def c_host(self):
        """The fb_csr_host view (the arrays must outlive the call)."""
        return _lib.CsrHost(self.shape[0], self.shape[1], self.val.size,
                            self.row_ptr.ctypes.data_as(C.c_void_p), self.col_ind.ctypes.data_as(C.c_void_p),
                            self.val.ctypes.data_as(C.c_void_p))


class UnitFilter:
    """UnitFilter<double, Index>: Dirichlet DOF indices and their values."""

    def __init__(self, indices, values=None):
        self.indices = np.ascontiguousarray(indices, dtype=np.uint64)
        self.values = (np.zeros(self.indices.size) if values is None
                       else np.ascontiguousarray(values, dtype=np.float64))

    def used_elements(self):
        return int(self.indices.size)

    def filter_rhs(self, v: DenseVector):
        v.elements[self.indices.astype(np.int64)] = self.values

    filter_sol = filter_rhs

    def filter_def(self, v: DenseVector):
        v.elements[self.indices.astype(np.int64)] = 0.0

    filter_cor = filter_def


class Transfer:
    """Transfer<SparseMatrixCSR>: prolongation (fine <- coarse) and restriction (coarse <- fine)."""

    def __init__(self, prol: SparseMatrixCSR, rest: SparseMatrixCSR = None):
        self.prol = prol
        self.rest = rest if rest is not None else prol.transpose()

    def get_mat_prol(self):
        return self.prol

    def get_mat_rest(self):
        return self.rest


# ------------------------------------------------------------------------------ Arch seam
def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class arch:
    """LAFEM::Arch drop-ins on CUDA tensors (kernel/lafem/arch/*.hpp)."""

    @staticmethod
    def apply_csr(r, a, x, b, y, val, col_ind, row_ptr, columns, transposed=False, stream=None):
        import torch
        rows = row_ptr.numel() - 1
        f = {(torch.float64, torch.int64): "fb_apply_csr_f64_u64", (torch.float64, torch.int32): "fb_apply_csr_f64_u32",
             (torch.float32, torch.int64): "fb_apply_csr_f32_u64",
             (torch.float32, torch.int32): "fb_apply_csr_f32_u32"}[(val.dtype, col_ind.dtype)]
        fn = getattr(_lib.lib(), f)
        _lib.check(fn(_ptr(r), a, _ptr(x), b, _ptr(y), _ptr(val), _ptr(col_ind), _ptr(row_ptr), rows, columns,
                      val.numel(), 1 if transposed else 0, _stream(stream)), f)

    @staticmethod
    def axpy(r, a, x, y, stream=None):
        fn = "fb_axpy_f64" if r.dtype.itemsize == 8 else "fb_axpy_f32"
        _lib.check(getattr(_lib.lib(), fn)(_ptr(r), a, _ptr(x), _ptr(y), r.numel(), _stream(stream)), fn)

    @staticmethod
    def dot(x, y, stream=None):
        f64 = x.dtype.itemsize == 8
        out = C.c_double() if f64 else C.c_float()
        fn = "fb_dot_f64" if f64 else "fb_dot_f32"
        _lib.check(getattr(_lib.lib(), fn)(C.byref(out), _ptr(x), _ptr(y), x.numel(), _stream(stream)), fn)
        return out.value

    @staticmethod
    def norm2(x, stream=None):
        f64 = x.dtype.itemsize == 8
        out = C.c_double() if f64 else C.c_float()
        fn = "fb_norm2_f64" if f64 else "fb_norm2_f32"
        _lib.check(getattr(_lib.lib(), fn)(C.byref(out), _ptr(x), x.numel(), _stream(stream)), fn)
        return out.value

    @staticmethod
    def component_product(r, x, y, stream=None):
        fn = "fb_component_product_f64" if r.dtype.itemsize == 8 else "fb_component_product_f32"
        _lib.check(getattr(_lib.lib(), fn)(_ptr(r), _ptr(x), _ptr(y), r.numel(), _stream(stream)), fn)

    @staticmethod
    def component_invert(r, x, s, stream=None):
        fn = "fb_component_invert_f64" if r.dtype.itemsize == 8 else "fb_component_invert_f32"
        _lib.check(getattr(_lib.lib(), fn)(_ptr(r), _ptr(x), s, r.numel(), _stream(stream)), fn)

    @staticmethod
    def scale(r, x, s, stream=None):
        fn = "fb_scale_f64" if r.dtype.itemsize == 8 else "fb_scale_f32"
        _lib.check(getattr(_lib.lib(), fn)(_ptr(r), _ptr(x), s, r.numel(), _stream(stream)), fn)

    @staticmethod
    def unit_filter_rhs(v, vals, idx, stream=None):
        fn = "fb_unit_filter_rhs_f64_u64" if v.dtype.itemsize == 8 else "fb_unit_filter_rhs_f32_u32"
        _lib.check(getattr(_lib.lib(), fn)(_ptr(v), _ptr(vals), _ptr(idx), idx.numel(), _stream(stream)), fn)

    @staticmethod
    def unit_filter_def(v, idx, stream=None):
        fn = "fb_unit_filter_def_f64_u64" if v.dtype.itemsize == 8 else "fb_unit_filter_def_f32_u32"
        _lib.check(getattr(_lib.lib(), fn)(_ptr(v), _ptr(idx), idx.numel(), _stream(stream)), fn)

    @staticmethod
    def diagonal_csr(diag, col_ind, row_ptr, stream=None):
        _lib.check(_lib.lib().fb_diagonal_csr_u64(_ptr(diag), _ptr(col_ind), _ptr(row_ptr), row_ptr.numel() - 1,
                                                   _stream(stream)), "fb_diagonal_csr_u64")

    @staticmethod
    def convert(dst, src, stream=None):
        fn = "fb_convert_f64_to_f32" if src.dtype.itemsize == 8 else "fb_convert_f32_to_f64"
        _lib.check(getattr(_lib.lib(), fn)(_ptr(dst), _ptr(src), src.numel(), _stream(stream)), fn)
