"""Q1 assembly on the device for the 2D unit-square family (fb_q1_pattern_2d, fb_q1_assemble_2d) and
the Laplacian on the unit cube (fb_q1_pattern_3d, fb_q1_assemble_3d, fb_q1_prolongation_3d).

The same operators as ``featb200.assembly`` (stiffness of -div(kappa grad u) with the 3x3 Gauss
rule, load vector of a sum of Gaussians, lexicographic vertices, Dirichlet entries of the load
vector zeroed), computed by CUDA kernels so that a parametric family of systems can be set up on
the GPU and handed to ``PCG.update_matrix`` without a host round trip.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def q1_pattern_2d(level):
    """(row_ptr, col_ind) of the row-sorted 9-point pattern of level `level` (numpy uint64)."""
    L = _lib.lib()
    nnz = C.c_uint64(0)
    _lib.check(L.fb_q1_pattern_2d(int(level), C.byref(nnz), None, None), "fb_q1_pattern_2d")
    n = (2 ** level + 1) ** 2
    rp = np.zeros(n + 1, dtype=np.uint64)
    ci = np.zeros(int(nnz.value), dtype=np.uint64)
    _lib.check(L.fb_q1_pattern_2d(int(level), C.byref(nnz), rp.ctypes.data_as(C.c_void_p),
                                  ci.ctypes.data_as(C.c_void_p)), "fb_q1_pattern_2d")
    return rp, ci


class Q1Assembler2D:
    """Device assembly of level `level`: ``assemble(field, gauss)`` returns CUDA float64 tensors
    (values in the q1_pattern_2d order, load vector)."""

    def __init__(self, level, device="cuda"):
        import torch
        self.level = int(level)
        self.row_ptr, self.col_ind = q1_pattern_2d(level)
        self.n = self.row_ptr.size - 1
        self.nnz = self.col_ind.size
        self.device = device
        self.row_ptr_d = torch.tensor(self.row_ptr.astype(np.int64), device=device)

    def assemble(self, field=None, gauss=None, values=True, rhs=True, stream=None, out_values=None, out_rhs=None):
        """field: None (kappa = 1) or featb200.assembly.field_params(...) (kx, ky, xi, eta, s) or the
        same with xi, eta as CUDA tensors; gauss: [g, 4] rows (c_x, c_y, w, a) or None (f = 0)."""
        import torch
        if stream is None:
            stream = torch.cuda.current_stream()
        dev = self.device
        vals = None
        b = None
        if values:
            vals = out_values if out_values is not None else torch.empty(self.nnz, dtype=torch.float64, device=dev)
        if rhs:
            b = out_rhs if out_rhs is not None else torch.empty(self.n, dtype=torch.float64, device=dev)
        k = 0
        xi_d = eta_d = None
        s = 0.0
        if field is not None and values:
            kx, ky, xi, eta, s = field
            k = int(len(kx))
            if not (np.array_equal(np.asarray(kx), np.arange(k) - k // 2) and np.array_equal(np.asarray(ky), np.asarray(kx))):
                raise ValueError("wave numbers must be -K/2 .. K/2-1 in both directions")
            xi_d = xi if torch.is_tensor(xi) else torch.tensor(np.ascontiguousarray(xi), dtype=torch.float64, device=dev)
            eta_d = eta if torch.is_tensor(eta) else torch.tensor(np.ascontiguousarray(eta), dtype=torch.float64, device=dev)
        ng = 0
        g_d = None
        if gauss is not None and rhs:
            g_d = gauss if torch.is_tensor(gauss) else torch.tensor(np.ascontiguousarray(gauss, dtype=np.float64),
                                                                    device=dev)
            if g_d.ndim != 2 or g_d.shape[1] != 4:
                raise ValueError("gauss rows must be (c_x, c_y, w, a)")
            ng = int(g_d.shape[0])
        elif rhs:
            b.zero_()
            if not values:
                return None, b
            rhs = False

        def ptr(t):
            return C.c_void_p(t.data_ptr()) if t is not None else None

        _lib.check(_lib.lib().fb_q1_assemble_2d(self.level, k, ptr(xi_d), ptr(eta_d), float(s), ng, ptr(g_d),
                                                ptr(self.row_ptr_d), ptr(vals), ptr(b) if rhs else None,
                                                C.c_void_p(stream.cuda_stream)), "fb_q1_assemble_2d")
        return vals, b


def sample_2d(level, field=None, gauss=None, stream=None, device="cuda"):
    """(f, g) at the vertices of level `level` as CUDA float64 tensors of (2^level+1)^2 entries:
    f = sum of the Gaussians (zeros without), g = log kappa of the field (zeros without)."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    n = (2 ** level + 1) ** 2
    f = torch.zeros(n, dtype=torch.float64, device=device)
    g = torch.zeros(n, dtype=torch.float64, device=device)
    k = 0
    s = 0.0
    xi_d = eta_d = g_d = None
    if field is not None:
        kx, ky, xi, eta, s = field
        k = int(len(kx))
        if not (np.array_equal(np.asarray(kx), np.arange(k) - k // 2) and np.array_equal(np.asarray(ky), np.asarray(kx))):
            raise ValueError("wave numbers must be -K/2 .. K/2-1 in both directions")
        xi_d = torch.tensor(np.ascontiguousarray(xi), dtype=torch.float64, device=device)
        eta_d = torch.tensor(np.ascontiguousarray(eta), dtype=torch.float64, device=device)
    ng = 0
    if gauss is not None:
        g_d = torch.tensor(np.ascontiguousarray(gauss, dtype=np.float64), device=device)
        ng = int(g_d.shape[0])
    if k == 0 and ng == 0:
        return f, g

    def ptr(t):
        return C.c_void_p(t.data_ptr()) if t is not None else None

    _lib.check(_lib.lib().fb_q1_sample_2d(int(level), k, ptr(xi_d), ptr(eta_d), float(s), ng, ptr(g_d),
                                          ptr(f) if ng else None, ptr(g) if k else None,
                                          C.c_void_p(stream.cuda_stream)), "fb_q1_sample_2d")
    return f, g


def q1_prolongation_2d(level, device="cuda", stream=None):
    """(row_ptr, col_ind, values) of the Q1 prolongation level-1 -> level as CUDA tensors
    (int64, int64, float64)."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    nnz = C.c_uint64(0)
    _lib.check(_lib.lib().fb_q1_prolongation_2d(int(level), C.byref(nnz), None, None, None, None),
               "fb_q1_prolongation_2d")
    n = (2 ** level + 1) ** 2
    rp = torch.empty(n + 1, dtype=torch.int64, device=device)
    ci = torch.empty(int(nnz.value), dtype=torch.int64, device=device)
    v = torch.empty(int(nnz.value), dtype=torch.float64, device=device)
    _lib.check(_lib.lib().fb_q1_prolongation_2d(int(level), C.byref(nnz), C.c_void_p(rp.data_ptr()),
                                                C.c_void_p(ci.data_ptr()), C.c_void_p(v.data_ptr()),
                                                C.c_void_p(stream.cuda_stream)), "fb_q1_prolongation_2d")
    return rp, ci, v


def q1_pattern_3d(level):
    """(row_ptr, col_ind) of the row-sorted 27-point pattern of the unit cube at `level` (numpy
    uint64; host code)."""
    L = _lib.lib()
    nnz = C.c_uint64(0)
    _lib.check(L.fb_q1_pattern_3d(int(level), C.byref(nnz), None, None), "fb_q1_pattern_3d")
    n = (2 ** level + 1) ** 3
    rp = np.zeros(n + 1, dtype=np.uint64)
    ci = np.zeros(int(nnz.value), dtype=np.uint64)
    _lib.check(L.fb_q1_pattern_3d(int(level), C.byref(nnz), rp.ctypes.data_as(C.c_void_p),
                                  ci.ctypes.data_as(C.c_void_p)), "fb_q1_pattern_3d")
    return rp, ci


class Q1Assembler3D:
    """Device assembly of the Laplacian on the unit cube at `level` (hexahedral Q1, lexicographic
    vertices): ``assemble(gauss)`` returns CUDA float64 tensors (stiffness values in the
    q1_pattern_3d order, load vector of the Gaussians with rows (c_x, c_y, c_z, w, a), boundary
    entries zeroed)."""

    def __init__(self, level, device="cuda"):
        import torch
        self.level = int(level)
        self.row_ptr, self.col_ind = q1_pattern_3d(level)
        self.n = self.row_ptr.size - 1
        self.nnz = self.col_ind.size
        self.device = device
        self.row_ptr_d = torch.tensor(self.row_ptr.astype(np.int64), device=device)

    def assemble(self, gauss=None, values=True, rhs=True, stream=None):
        import torch
        if stream is None:
            stream = torch.cuda.current_stream()
        vals = torch.empty(self.nnz, dtype=torch.float64, device=self.device) if values else None
        b = torch.zeros(self.n, dtype=torch.float64, device=self.device) if rhs else None
        g_d = None
        ng = 0
        if gauss is not None and rhs:
            g_d = torch.tensor(np.ascontiguousarray(gauss, dtype=np.float64), device=self.device)
            if g_d.ndim != 2 or g_d.shape[1] != 5:
                raise ValueError("gauss rows must be (c_x, c_y, c_z, w, a)")
            ng = int(g_d.shape[0])
        elif rhs and not values:
            return None, b

        def ptr(t):
            return C.c_void_p(t.data_ptr()) if t is not None else None

        _lib.check(_lib.lib().fb_q1_assemble_3d(self.level, ng, ptr(g_d), ptr(self.row_ptr_d), ptr(vals),
                                                ptr(b) if (rhs and ng) else None, C.c_void_p(stream.cuda_stream)),
                   "fb_q1_assemble_3d")
        return vals, b


def q1_prolongation_3d(level, device="cuda", stream=None):
    """(row_ptr, col_ind, values) of the 3D Q1 prolongation level-1 -> level as CUDA tensors
    (int64, int64, float64)."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    nnz = C.c_uint64(0)
    _lib.check(_lib.lib().fb_q1_prolongation_3d(int(level), C.byref(nnz), None, None, None, None),
               "fb_q1_prolongation_3d")
    n = (2 ** level + 1) ** 3
    rp = torch.empty(n + 1, dtype=torch.int64, device=device)
    ci = torch.empty(int(nnz.value), dtype=torch.int64, device=device)
    v = torch.empty(int(nnz.value), dtype=torch.float64, device=device)
    _lib.check(_lib.lib().fb_q1_prolongation_3d(int(level), C.byref(nnz), C.c_void_p(rp.data_ptr()),
                                                C.c_void_p(ci.data_ptr()), C.c_void_p(v.data_ptr()),
                                                C.c_void_p(stream.cuda_stream)), "fb_q1_prolongation_3d")
    return rp, ci, v
