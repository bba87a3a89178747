"""Learned warm start for a parametric family of Poisson problems.

Family: -div(kappa grad u) = f on the unit square, Q1 on the uniformly refined mesh of level
`level` (homogeneous Dirichlet boundary), kappa = exp(g) with g a seeded 16x16-mode Gaussian random
field (spectral decay |k|^-2, std 1), f a sum of 8 seeded Gaussians.  Instance k uses
``assembly.gauss_params(seed_base + 2k)`` and ``assembly.field_params(seed_base + 2k + 1)``.

Pipeline (all on the GPU): the levels' matrices and the load vector are assembled by the library
(fb_q1_assemble_2d) into one solver (fb_solver_update_matrix); the network input is (f, log kappa)
sampled at the vertices of level `net_level` (fb_q1_sample_2d); the network (fb_unet_*) predicts u
there; the prediction is carried to the finest level by nested iteration (the hierarchy's own
transfer matrices, then damped Jacobi on each finer level against the restricted load vector, all
through the library's LAFEM::Arch kernels) and used as the PCG initial guess.  The stopping test is the same for every start:
||d|| <= tol * ||b|| (the zero guess's initial defect), so a better start saves iterations.  A
start whose defect is not smaller than ||b|| falls back to zero.
"""
from __future__ import annotations

import time

import numpy as np

from . import assembly as AS
from .assembly_gpu import Q1Assembler2D, sample_2d
from .lafem import arch
from .solver import Status, build_pcg_multigrid
from .unet import UNet

SEED_BASE = 1_000_000


class ParametricFamily:
    def __init__(self, level=9, net_level=7, precision="f64", ordering="native", seed_base=SEED_BASE, tol=1e-8):
        import torch
        if net_level >= level or net_level < 3:
            raise ValueError("need 3 <= net_level < level")
        self.level, self.net_level = int(level), int(net_level)
        self.G = 2 ** net_level + 1
        self.seed_base = int(seed_base)
        self.tol = float(tol)
        levels, _ = AS.poisson_hierarchy(level, 2, rhs="sine")
        self.levels = levels
        self.solver = build_pcg_multigrid(levels, precision=precision, ordering=ordering, max_iter=100)
        self.asm = [Q1Assembler2D(L["level"]) for L in levels]
        dev = "cuda"
        self.omega, self.smooth_steps, self.smooth_net = 0.7, 2, 8

        def dev_csr(M):
            return (torch.tensor(M.val, device=dev), torch.tensor(M.col_ind.astype(np.int64), device=dev),
                    torch.tensor(M.row_ptr.astype(np.int64), device=dev), M.columns(), M.rows())

        # levels 0 .. nfine-1 (finest first) are the ones above the network grid
        self.nfine = level - net_level
        self.P = [dev_csr(levels[i]["transfer"].get_mat_prol()) for i in range(self.nfine)]
        self.R = [dev_csr(levels[i]["transfer"].get_mat_rest()) for i in range(self.nfine)]
        self.A_pat = []
        self.diag_pos = []
        for i in range(self.nfine + 1):
            A = levels[i]["matrix"]
            col = torch.tensor(A.col_ind.astype(np.int64), device=dev)
            rp = torch.tensor(A.row_ptr.astype(np.int64), device=dev)
            pos = torch.empty(A.rows(), dtype=torch.int64, device=dev)
            arch.diagonal_csr(pos, col, rp)
            self.A_pat.append((col, rp, A.rows()))
            self.diag_pos.append(pos)
        self.fidx_l = [torch.tensor(levels[i]["filter"].indices.astype(np.int64), device=dev)
                       for i in range(self.nfine + 1)]
        self.fidx = self.fidx_l[0]
        self.A_col, self.A_rp, self.n = self.A_pat[0]
        self.vals = [None] * (self.nfine + 1)
        self.A_val = None
        self.b = None

    # ------------------------------------------------------------------ instances
    def params(self, k):
        s = self.seed_base + 2 * int(k)
        return AS.field_params(s + 1), AS.gauss_params(s, 2)

    def setup(self, k):
        """Assemble instance k on the device and load it into the solver; returns b (CUDA)."""
        fp, gp = self.params(k)
        for l, L in enumerate(self.levels):
            vals, b = self.asm[l].assemble(fp, gp if l == 0 else None, rhs=(l == 0))
            self.solver.update_matrix(l, vals)
            if l <= self.nfine:
                self.vals[l] = vals
            if l == 0:
                self.b = b
        self.A_val = self.vals[0]
        return self.b

    def net_input(self, k):
        """(f, log kappa) at the network grid's vertices, float32 [2, G, G] (CUDA)."""
        import torch
        fp, gp = self.params(k)
        f, g = sample_2d(self.net_level, fp, gp)
        return torch.stack([f, g]).view(2, self.G, self.G).float()

    def restrict_solution(self, u):
        """u (finest level, lexicographic) at the network grid's vertices (injection)."""
        N = 2 ** self.level + 1
        s = 2 ** (self.level - self.net_level)
        return u.view(N, N)[::s, ::s]

    # ------------------------------------------------------------------ solves
    def solve(self, x):
        """PCG-MG from the initial guess in x (overwritten by the solution), stop at
        ||d|| <= tol ||b||; returns (status, iterations)."""
        nb = arch.norm2(self.b)
        self.solver.set_tolerances(1.0, self.tol * nb)
        st = self.solver.correct_device(x, self.b)
        return st, self.solver.get_num_iter()

    def _jacobi(self, i, x, b, steps):
        """`steps` damped-Jacobi steps x += omega D^-1 F(b - A x) on level index i (library kernels)."""
        import torch
        col, rp, n = self.A_pat[i]
        vals = self.vals[i]
        dinv = torch.empty(n, dtype=torch.float64, device=x.device)
        arch.component_invert(dinv, vals.index_select(0, self.diag_pos[i]), self.omega)
        r = torch.empty_like(x)
        for _ in range(steps):
            arch.apply_csr(r, -1.0, x, 1.0, b, vals, col, rp, n)
            arch.unit_filter_def(r, self.fidx_l[i])
            arch.component_product(r, dinv, r)
            arch.axpy(x, 1.0, r, x)

    def prolongate(self, u_net, smooth=None):
        """Network-grid values (float32/float64 [G, G]) -> finest-level initial guess (float64) by
        nested iteration: smooth on the network's grid (`smooth_net` damped-Jacobi steps, which damp
        the prediction's grid-scale noise), then on every finer level prolongate (the hierarchy's P),
        zero the Dirichlet values and take `smooth` damped-Jacobi steps, each level against its
        right-hand side (the restricted load vector)."""
        import torch
        steps = self.smooth_steps if smooth is None else int(smooth)
        dev = u_net.device
        # right-hand sides down to the network grid: b_{i+1} = F(R_i b_i)
        bl = [self.b]
        for i in range(self.nfine):
            val, col, rp, cols, rows = self.R[i]
            bc = torch.empty(rows, dtype=torch.float64, device=dev)
            arch.apply_csr(bc, 1.0, bl[-1], 0.0, None, val, col, rp, cols)
            arch.unit_filter_def(bc, self.fidx_l[i + 1])
            bl.append(bc)
        x = u_net.reshape(-1).to(torch.float64).contiguous()
        arch.unit_filter_def(x, self.fidx_l[self.nfine])
        if self.smooth_net:
            self._jacobi(self.nfine, x, bl[self.nfine], self.smooth_net)
        for i in range(self.nfine - 1, -1, -1):
            val, col, rp, cols, rows = self.P[i]
            y = torch.empty(rows, dtype=torch.float64, device=dev)
            arch.apply_csr(y, 1.0, x, 0.0, None, val, col, rp, cols)
            arch.unit_filter_def(y, self.fidx_l[i])
            if steps:
                self._jacobi(i, y, bl[i], steps)
            x = y
        return x

    def defect_norm(self, x):
        """||F(b - A x)|| on the finest level."""
        import torch
        r = torch.empty_like(self.b)
        arch.apply_csr(r, -1.0, x, 1.0, self.b, self.A_val, self.A_col, self.A_rp, self.n)
        arch.unit_filter_def(r, self.fidx)
        return arch.norm2(r)

    # ------------------------------------------------------------------ data
    def generate(self, indices, log_every=0):
        """Training pairs for the instances `indices`: inputs [N, 2, G, G] (f, log kappa) and targets
        [N, G, G] (the FP64-multigrid solution at the network grid), float32 CUDA tensors; plus the
        zero-guess iteration counts."""
        import torch
        indices = list(indices)
        N = len(indices)
        X = torch.empty((N, 2, self.G, self.G), dtype=torch.float32, device="cuda")
        Y = torch.empty((N, self.G, self.G), dtype=torch.float32, device="cuda")
        its = np.zeros(N, dtype=np.int64)
        x = torch.empty(self.n, dtype=torch.float64, device="cuda")
        t0 = time.time()
        for j, k in enumerate(indices):
            self.setup(k)
            X[j] = self.net_input(k)
            x.zero_()
            st, it = self.solve(x)
            if st != Status.success:
                raise RuntimeError(f"instance {k}: solve status {st!r}")
            its[j] = it
            Y[j] = self.restrict_solution(x).float()
            if log_every and (j + 1) % log_every == 0:
                print(f"generated {j + 1}/{N} ({time.time() - t0:.1f} s)", flush=True)
        return X, Y, its


class WarmStart:
    """The trained network with its input/output scaling."""

    def __init__(self, family: ParametricFamily, max_batch=32, seed=0):
        self.family = family
        self.net = UNet(family.G, max_batch, seed=seed)
        self.u_scale = 1.0

    @staticmethod
    def _f_norm(f):
        """Per-instance scale of the load (RMS over the grid): u is linear in f for a fixed kappa,
        so the network sees f / |f| and predicts u / |f|."""
        return f.pow(2).mean(dim=(-2, -1)).sqrt().clamp_min(1e-30)

    def fit(self, X, Y, epochs=10, batch=32, lr=2e-3, log_every=0, seed=0):
        """Adam on the MSE of the normalised target with cosine learning-rate decay; returns the
        per-epoch mean training loss."""
        import torch
        sig = self._f_norm(X[:, 0])[:, None, None]
        Xs = X.clone()
        Xs[:, 0] /= sig
        Yn = Y / sig
        self.u_scale = float(1.0 / max(Yn.std().item(), 1e-30))
        Ys = Yn * self.u_scale
        N = X.shape[0]
        rng = np.random.default_rng(seed)
        g = torch.empty((batch, self.family.G, self.family.G), dtype=torch.float32, device="cuda")
        steps = epochs * (N // batch)
        hist = []
        t = 0
        for ep in range(epochs):
            perm = torch.tensor(rng.permutation(N), device="cuda")
            losses = []
            for i in range(N // batch):
                idx = perm[i * batch:(i + 1) * batch]
                xb = Xs.index_select(0, idx).contiguous()
                yb = Ys.index_select(0, idx).contiguous()
                cur = lr * 0.5 * (1.0 + np.cos(np.pi * t / max(steps, 1)))
                losses.append(self.net.train_step(xb, yb, cur, g).clone())
                t += 1
            hist.append(float(torch.cat(losses).mean().item()) if losses else float("nan"))
            if log_every:
                print(f"epoch {ep + 1}/{epochs}: loss {hist[-1]:.4e}", flush=True)
        return hist

    def predict(self, inp):
        """inp [2, G, G] unscaled -> u at the network grid (float32 [G, G])."""
        x = inp.clone()
        sig = self._f_norm(x[0])
        x[0] /= sig
        y = self.net.forward(x.unsqueeze(0).contiguous())
        return y[0] * (sig / self.u_scale)

    def initial_guess(self, k, fallback=True):
        """(x0, used_network, ||d_0|| / ||b||): the prolongated prediction, or zeros when its defect
        is not below ||b|| (fallback=False keeps the prediction regardless)."""
        import torch
        fam = self.family
        x0 = fam.prolongate(self.predict(fam.net_input(k)))
        ratio = fam.defect_norm(x0) / max(arch.norm2(fam.b), 1e-300)
        if ratio < 1.0 or not fallback:
            return x0, True, ratio
        return torch.zeros_like(x0), False, ratio


def evaluate(ws: WarmStart, indices, fallback=True):
    """Per instance: iterations and device-synchronised ms (assembly excluded) of the zero-guess
    solve and of the warm-started solve (network inference, prolongation and the fallback test
    included), whether the network start was used, and the relative difference of the two
    solutions."""
    import torch
    fam = ws.family
    rows = []
    for k in indices:
        fam.setup(k)
        torch.cuda.synchronize()
        x = torch.zeros(fam.n, dtype=torch.float64, device="cuda")
        t0 = time.perf_counter()
        st0, it0 = fam.solve(x)
        torch.cuda.synchronize()
        ms0 = (time.perf_counter() - t0) * 1e3
        t1 = time.perf_counter()
        x0, used, ratio = ws.initial_guess(k, fallback)
        st1, it1 = fam.solve(x0)
        torch.cuda.synchronize()
        ms1 = (time.perf_counter() - t1) * 1e3
        diff = float((x0 - x).norm().item() / max(x.norm().item(), 1e-300))
        rows.append({"k": int(k), "it_zero": int(it0), "it_warm": int(it1), "ms_zero": ms0, "ms_warm": ms1,
                     "used": bool(used), "d0_ratio": float(ratio),
                     "ok": st0 == Status.success and st1 == Status.success, "rel_diff": diff})
    return rows
