"""Synthetic Poisson problems on the unit square / cube: Q1 finite elements on uniformly refined
quadrilateral / hexahedral meshes, lexicographic vertex numbering.

This is set-up code (it runs once, on the host) that produces the inputs of the solve path in the
layout of the reference's assembly: the Laplace (or kappa-weighted Laplace) stiffness matrix
assembled with the tensor Gauss-Legendre rule the reference selects for "auto-degree:5"
(3 points per direction, kernel/cubature/auto_alias.hpp), the Q1 prolongation
(kernel/assembly/grid_transfer.hpp, assemble_prolongation_direct) with R = P^T, unit filters on
the whole boundary, and load vectors of the form int f phi_i.  The reference numbers vertices
hierarchically (kernel/geometry/intern/standard_vertex_refiner.hpp:190-225); the matrices here are
the same operators in a lexicographic numbering.

Random coefficients (Gaussian right-hand sides, log-normal kappa fields) come from numpy's seeded
PCG64 generator; ``write_params`` stores them in the text form the reference-side driver reads, so
both sides consume identical coefficients.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .lafem import SparseMatrixCSR, Transfer, UnitFilter

GL3_X = np.array([-np.sqrt(3.0 / 5.0), 0.0, np.sqrt(3.0 / 5.0)])
GL3_W = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])


# ------------------------------------------------------------------------------ coefficients
def gauss_params(seed, dim=2, count=8, width=(0.02, 0.1)):
    """count Gaussians: centres U[0.1,0.9]^dim, widths U[width], amplitudes N(0,1).
    Rows: c_1..c_dim, w, a."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.1, 0.9, size=(count, dim))
    w = rng.uniform(width[0], width[1], size=count)
    a = rng.standard_normal(count)
    return np.column_stack([c, w, a])


def gauss_eval(params, *xs):
    dim = len(xs)
    out = np.zeros(np.broadcast(*xs).shape)
    for row in params:
        r2 = sum((xs[d] - row[d]) ** 2 for d in range(dim))
        out += row[dim + 1] * np.exp(-r2 / (2.0 * row[dim] ** 2))
    return out


def field_params(seed, k=16):
    """Gaussian random field g = s sum (xi cos t + eta sin t)/|k|^2 over wave vectors
    k in {-k/2..k/2-1}^2 without 0, t = 2 pi (kx x + ky y), s normalising Var g to 1.
    Returns (kx, ky, xi[k,k], eta[k,k], s)."""
    rng = np.random.default_rng(seed)
    kv = np.arange(k, dtype=np.float64) - k // 2
    xi = rng.standard_normal((k, k))
    eta = rng.standard_normal((k, k))
    den = kv[:, None] ** 2 + kv[None, :] ** 2
    inv4 = np.where(den > 0, 1.0 / np.where(den > 0, den, 1.0) ** 2, 0.0)
    s = 1.0 / np.sqrt(inv4.sum())
    return kv.copy(), kv.copy(), xi, eta, s


def field_eval_grid(fp, xs, ys):
    """g on the tensor grid xs (nx) x ys (ny) -> array [ny, nx] (separable evaluation)."""
    kx, ky, xi, eta, s = fp
    den = kx[:, None] ** 2 + ky[None, :] ** 2
    safe = np.where(den > 0, den, 1.0)
    c = np.where(den > 0, (xi - 1j * eta) / safe, 0.0)                # [i, j]
    ey = np.exp(2j * np.pi * ky[:, None] * ys[None, :])               # [j, ny]
    h = c @ ey                                                        # [i, ny]
    ex = np.exp(2j * np.pi * kx[:, None] * xs[None, :])               # [i, nx]
    return s * np.real(h.T @ ex)                                      # [ny, nx]


def write_params(path, gauss=None, field=None):
    """Text files for the reference-side driver (--params / --kappa)."""
    if gauss is not None:
        np.savetxt(path, gauss, fmt="%.17g")
    if field is not None:
        kx, ky, xi, eta, s = field
        with open(path, "w") as f:
            f.write(f"{kx.size} {float(s)!r}\n")
            for v in kx:
                f.write(f"{float(v)!r}\n")
            for v in ky:
                f.write(f"{float(v)!r}\n")
            for a, b in zip(xi.ravel(), eta.ravel()):
                f.write(f"{float(a)!r} {float(b)!r}\n")


# ------------------------------------------------------------------------------ Q1 assembly
def _q1_ref(dim):
    """Reference-element data at the 3^dim Gauss points: values [q, v], grads [q, v, d], weights [q]."""
    pts = np.array(np.meshgrid(*([GL3_X] * dim), indexing="ij")).reshape(dim, -1).T   # [q, d]
    w = np.prod(np.array(np.meshgrid(*([GL3_W] * dim), indexing="ij")).reshape(dim, -1).T, axis=1)
    nv = 2 ** dim
    signs = np.array([[1.0 if (v >> d) & 1 else -1.0 for d in range(dim)] for v in range(nv)])  # [v, d]
    fac = 1.0 + pts[:, None, :] * signs[None, :, :]                    # [q, v, d]
    val = np.prod(fac, axis=2) / nv
    grad = np.empty((pts.shape[0], nv, dim))
    for d in range(dim):
        others = np.prod(np.delete(fac, d, axis=2), axis=2) if dim > 1 else 1.0
        grad[:, :, d] = signs[None, :, d] * others / nv
    return pts, w, val, grad


def _cells(level, dim):
    N = 2 ** level
    idx = np.indices((N,) * dim).reshape(dim, -1)                      # [d, cells], d=0 is x
    nvx = N + 1
    strides = np.array([nvx ** d for d in range(dim)])
    base = (idx * strides[:, None]).sum(axis=0)
    offs = np.array([sum(((v >> d) & 1) * strides[d] for d in range(dim)) for v in range(2 ** dim)])
    return base[:, None] + offs[None, :], idx                            # [cells, v]


def _vertex_coords(level, dim):
    N = 2 ** level
    g = np.indices((N + 1,) * dim)[::-1].reshape(dim, -1)              # d=0 (x) fastest
    return g.T / N


def stiffness(level, dim=2, kappa=None):
    """Q1 stiffness of -div(kappa grad u) on the unit square/cube at `level` (CSR, sorted).
    kappa: None or a callable on quadrature-point coordinate arrays (x, y[, z]) -> values."""
    N = 2 ** level
    h = 1.0 / N
    pts, w, val, grad = _q1_ref(dim)
    # physical gradient = grad * (2/h); det J = (h/2)^dim
    fac = (h / 2.0) ** dim * (2.0 / h) ** 2
    gg = np.einsum("qvd,qud->qvu", grad, grad)                          # [q, v, u]
    conn, idx = _cells(level, dim)
    nverts = (N + 1) ** dim
    if kappa is None:
        kloc = fac * np.einsum("q,qvu->vu", w, gg)
        data = np.broadcast_to(kloc, (conn.shape[0],) + kloc.shape)
    else:
        # quadrature coordinates of every cell: x_d = (idx_d + (1 + xi_d)/2) h
        xq = [(idx[d][:, None] + (1.0 + pts[None, :, d]) / 2.0) * h for d in range(dim)]
        kq = kappa(*xq)                                                  # [cells, q]
        data = fac * np.einsum("cq,q,qvu->cvu", kq, w, gg)
    rows = np.repeat(conn, conn.shape[1], axis=1).ravel()
    cols = np.tile(conn, (1, conn.shape[1])).ravel()
    A = sp.coo_matrix((np.asarray(data).ravel(), (rows, cols)), shape=(nverts, nverts)).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return A


def prolongation(level, dim=2):
    """Q1 prolongation level-1 -> level (lexicographic on both), weights 1, 1/2, 1/4, 1/8."""
    Nf = 2 ** level
    Nc = Nf // 2
    fine = np.indices((Nf + 1,) * dim)[::-1].reshape(dim, -1)          # [d, nf], d=0 (x) fastest
    rows, cols, vals = [], [], []
    nf = fine.shape[1]
    combos = [np.array([(c >> d) & 1 for d in range(dim)]) for c in range(2 ** dim)]
    for comb in combos:
        # coarse index per direction: even -> i/2 (one choice, comb bit must be 0); odd -> (i-1)/2 + bit
        ok = np.ones(nf, dtype=bool)
        cidx = np.zeros(nf, dtype=np.int64)
        wgt = np.ones(nf)
        for d in range(dim):
            i = fine[d]
            odd = (i & 1) == 1
            ok &= odd | (comb[d] == 0)
            ci = np.where(odd, (i - 1) // 2 + comb[d], i // 2)
            wgt = wgt * np.where(odd, 0.5, 1.0)
            cidx += ci * (Nc + 1) ** d
        sel = np.nonzero(ok)[0]
        rows.append(sel)
        cols.append(cidx[sel])
        vals.append(wgt[sel])
    P = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nf, (Nc + 1) ** dim)).tocsr()
    P.sort_indices()
    return P


def boundary_dofs(level, dim=2):
    N = 2 ** level
    g = np.indices((N + 1,) * dim)[::-1].reshape(dim, -1)
    on = np.zeros(g.shape[1], dtype=bool)
    for d in range(dim):
        on |= (g[d] == 0) | (g[d] == N)
    return np.nonzero(on)[0].astype(np.uint64)


def load_vector(level, f, dim=2):
    """b_i = int f phi_i with the 3^dim Gauss rule; f on coordinate arrays (x, y[, z])."""
    N = 2 ** level
    h = 1.0 / N
    pts, w, val, _ = _q1_ref(dim)
    conn, idx = _cells(level, dim)
    xq = [(idx[d][:, None] + (1.0 + pts[None, :, d]) / 2.0) * h for d in range(dim)]
    fq = f(*xq)                                                          # [cells, q]
    loc = (h / 2.0) ** dim * np.einsum("cq,q,qv->cv", fq, w, val)
    b = np.bincount(conn.ravel(), weights=loc.ravel(), minlength=(N + 1) ** dim)
    return b


def sine_bubble_rhs(*xs):
    """-Laplace of u = prod sin(pi x_d): dim * pi^2 * prod sin(pi x_d) (LaplaceFunctional of the
    SineBubbleFunction, kernel/analytic/common.hpp:376)."""
    dim = len(xs)
    out = dim * np.pi ** 2 * np.ones(np.broadcast(*xs).shape)
    for x in xs:
        out = out * np.sin(np.pi * x)
    return out


def poisson_hierarchy(level, dim=2, level_min=1, rhs="sine", gauss=None, field=None):
    """Finest-first list of levels (matrix, filter, transfer) and the filtered fine rhs."""
    kappa = None
    if field is not None:
        if dim != 2:
            raise ValueError("kappa fields are 2D")

        def kappa(x, y, _fp=field):
            # x, y: [cells, q]; evaluate on the tensor grid of the distinct coordinates
            xs = np.unique(x)
            ys = np.unique(y)
            G = field_eval_grid(_fp, xs, ys)
            ix = np.searchsorted(xs, x)
            iy = np.searchsorted(ys, y)
            return np.exp(G[iy, ix])
    levels = []
    for lv in range(level, level_min - 1, -1):
        A = SparseMatrixCSR.from_scipy(stiffness(lv, dim, kappa))
        fidx = boundary_dofs(lv, dim)
        d = {"matrix": A, "filter": UnitFilter(fidx), "level": lv}
        if lv > level_min:
            P = prolongation(lv, dim)
            d["transfer"] = Transfer(SparseMatrixCSR.from_scipy(P), SparseMatrixCSR.from_scipy(P.T.tocsr()))
        levels.append(d)
    if rhs == "sine":
        b = load_vector(level, sine_bubble_rhs, dim)
    elif rhs == "gauss":
        b = load_vector(level, lambda *xs: gauss_eval(gauss, *xs), dim)
    else:
        raise ValueError(rhs)
    b[levels[0]["filter"].indices.astype(np.int64)] = 0.0
    return levels, b


def vertex_coords(level, dim=2):
    return _vertex_coords(level, dim)


# ------------------------------------------------------------------------------ named workload families
def batch_family_levels(count=256, seed=7):
    """Levels of the uneven-instance batch: `count` draws uniform in 5..9 (seeded PCG64)."""
    return [int(v) for v in np.random.default_rng(seed).integers(5, 10, size=count)]


def batch_instance_params(k):
    """(Gaussian right-hand side, kappa field) of instance k of the uneven-instance batch."""
    return gauss_params(10_000 + 2 * k, 2), field_params(10_001 + 2 * k)


def batch_instance(level, k):
    """Instance k of the uneven-instance batch at `level`: -div(kappa grad u) = f with
    kappa = exp(16x16-mode random field) and an 8-Gaussian f; (levels, filtered rhs)."""
    g, f = batch_instance_params(k)
    return poisson_hierarchy(level, 2, rhs="gauss", gauss=g, field=f)


def gauss_load_vector(level, params, dim=2):
    """load_vector of the Gaussian sum `params` (gauss_params rows), formed by direction: each
    Gaussian, the Gauss rule and the Q1 basis factor into one factor per coordinate, so
    b = sum_k a_k (B_k,z (x) B_k,y (x) B_k,x) with B_k,d[i] the 1D load vector of the k-th Gaussian's
    factor in direction d.  The same integral as load_vector with gauss_eval, to rounding, in
    O(count x vertices) instead of O(count x cells x 3^dim)."""
    N = 2 ** level
    h = 1.0 / N
    e = np.arange(N)
    xq = (e[:, None] + (1.0 + GL3_X[None, :]) / 2.0) * h                # [cells, q], 1D
    phi = np.stack([(1.0 - GL3_X) / 2.0, (1.0 + GL3_X) / 2.0])          # [local vertex, q]
    b = np.zeros((N + 1,) * dim)
    for row in params:
        w, a = row[dim], row[dim + 1]
        term = None
        for d in range(dim):
            g = np.exp(-((xq - row[d]) ** 2) / (2.0 * w * w))            # [cells, q]
            loc = (h / 2.0) * np.einsum("cq,q,vq->cv", g, GL3_W, phi)
            B = np.zeros(N + 1)
            B[:-1] += loc[:, 0]
            B[1:] += loc[:, 1]
            # x fastest: direction d is axis dim-1-d of the vertex array
            shape = [1] * dim
            shape[dim - 1 - d] = N + 1
            term = B.reshape(shape) if term is None else term * B.reshape(shape)
        b += a * term
    return b.ravel()


def rhs64_params(j, dim=3):
    """Gaussian right-hand side j (0..63) of the many-right-hand-side 3D set (seeds 100..163)."""
    return gauss_params(100 + j, dim, width=(0.03, 0.12) if dim == 3 else (0.02, 0.1))


def rhs64_family(level=6, dim=3, k=64):
    """The many-right-hand-side set: the Q1 Poisson hierarchy at `level` and a [rows, k] array of
    filtered 8-Gaussian load vectors (column j from rhs64_params(j))."""
    levels, _ = poisson_hierarchy(level, dim, rhs="sine")
    fidx = levels[0]["filter"].indices.astype(np.int64)
    B = np.zeros((levels[0]["matrix"].rows(), k))
    for j in range(k):
        b = gauss_load_vector(level, rhs64_params(j, dim), dim)
        b[fidx] = 0.0
        B[:, j] = b
    return levels, B
