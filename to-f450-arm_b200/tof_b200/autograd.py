"""Differentiable SIMP objective over the design density (torch.autograd).

    J(x) = c(rho(x)) + P(rho(x))

* rho = the density filter of the design variables x on the design cells,
  1 on keep-solid cells (src/topopt.py:270-281; FILTER_PHYSICAL).
* c = sum_i w_i F_i^T u_i with K(rho) u_i = F_i (src/topopt.py:287-306),
  evaluated in the stationary form sum_i w_i (2 F_i^T u_i - u_i^T K u_i),
  equal to it at the exact solution and second-order in the solve error, so
  finite differences of J are not limited by the iterative solve (whose true
  residual floor in FP64 is ~1e-9 on high-contrast SIMP designs).
* P = 1/2 mu s lambda_t max(0, 1 - lambda / lambda_t)^2, lambda the tracked
  eigenvalue of K phi = lambda M phi (tip mass included), s = s_c / s_m the
  reference's sensitivity scale (src/topopt.py:340-361), held constant.  Its
  gradient is the reference's penalty term -mu s viol dlambda/drho.

The backward pass is hand-written (no autograd tape through the solvers):

    dJ/drho_e = dc/drho_e - mu s viol dlambda/drho_e
    dc/drho_e = -sum_i w_i p (1 - emin) rho_e^(p-1) u_e^T Ke u_e
                (self-adjoint compliance; libtof k_compliance_sens)
    dlambda/drho_e = (p (1 - emin) rho_e^(p-1) phi_e^T Ke phi_e
                      - lambda m'(rho_e) phi_e^T Me phi_e) / phi^T M phi
                (src/fem.py:472-526; libtof k_eig_sens)
    dJ/dx = F^T dJ/drho   (exact transpose of the density filter,
                           FILTER_ADJOINT)

The reference's own sensitivity instead filters dJ/drho with its normalised
average (src/topopt.py:311, 361); `reference_sensitivity()` returns that form
so it can be compared with the reference's analytic dc/dx.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L


class SIMPObjective:
    """J(x) of one design, built on a `tof_b200.topopt.SIMPOptimizer` (its
    context, filter, loads, weights, tip mass and frequency target).

    mu:          penalty weight (default: the optimiser's current mu);
    pcg_rtol:    static solve tolerance;
    modal_tol:   LOBPCG relative residual tolerance.
    The tracked mode is the lowest at the first evaluation; later evaluations
    (finite-difference neighbours) pick the mode with the largest MAC against
    it (src/topopt.py:179-188).  The scale s is fixed at the first evaluation
    where the frequency constraint is violated.
    """

    def __init__(self, opt, mu: float = None, pcg_rtol: float = 1e-8, modal_tol: float = 1e-6,
                 modal_maxiter: int = 2000):
        self.opt = opt
        self.ctx = opt.ctx
        self.mu = opt.mu_freq_cur if mu is None else float(mu)
        self.pcg_rtol, self.modal_tol, self.modal_maxiter = pcg_rtol, modal_tol, modal_maxiter
        self.mode_id = opt.fem._mode_id()
        self.v_ref = None
        self.scale = None
        self.X4 = None
        self.last = None

    # ------------------------------------------------------------------ #
    def _modal(self):
        opt, ctx = self.opt, self.ctx
        n = opt.n_modes_track
        nb = min(opt.fem.max_modes, n + 2)
        if self.X4 is None:
            n_free = len(opt.fem.free_dofs)
            X0 = np.random.default_rng(0).standard_normal((n_free, nb))
            full = np.zeros((nb, opt.geom.n_dofs))
            full[:, opt.fem.free_dofs] = X0.T
            self.X4 = ctx.pack(torch.from_numpy(full))
        precond = L.PRECOND_MG if self.mode_id == L.MODE_MIXED else L.PRECOND_JACOBI
        modes, lam, st = ctx.lobpcg(self.X4, n, tol=self.modal_tol, maxiter=self.modal_maxiter,
                                    mode=self.mode_id, precond=precond)
        # LOBPCG stops at the best iterate when its residual stalls (on the
        # softest SIMP designs the lowest modes stall near 1e-5); eigenvalues
        # are second-order in that residual, so a stall within 100x of the
        # tolerance is accepted, anything worse is an error
        if st["status"] < 0 or st["relres"] > 100.0 * self.modal_tol:
            raise L.SolverError("tof_lobpcg", st["status"],
                                f"modal solve stopped at residual {st['relres']:.2e} (tolerance {self.modal_tol:.1e})")
        self.modal_stats = st
        self.X4 = ctx.last_block                        # all final Ritz vectors: the next warm start
        return modes, np.maximum(lam, 0.0)

    def evaluate(self, x: torch.Tensor) -> dict:
        """J and dJ/drho at the design field x (full element grid, x fastest;
        only design cells are read)."""
        opt, ctx = self.opt, self.ctx
        x = x.to(ctx.device, torch.float64).contiguous()
        rho = opt.filter.apply(x, L.FILTER_PHYSICAL)
        ctx.set_density(rho)
        opt.fem._rho_dev = None
        if opt.modal_active:
            ctx.set_tip_lump(opt._tip3)
            opt.fem._tip_key = opt._tip_key
        u4, st = ctx.pcg(opt.b4, None, rtol=self.pcg_rtol, maxiter=20000, mode=self.mode_id)
        if any(s["status"] != L.TOF_OK for s in st):
            worst = max(s["relres"] for s in st)
            raise L.SolverError("tof_pcg", max(s["status"] for s in st),
                                f"static solve did not reach pcg_rtol (relres {worst:.2e})")
        ce = ctx.quadform(L.OP_K, u4)
        c_energy, dc = ctx.compliance_sens(ce, opt.w_dev)           # sum_i w_i u_i^T K u_i
        Fu = (opt.b4[:, :, :3] * u4[:, :, :3]).sum(dim=(1, 2))        # F_i^T u_i (fixed DOFs are 0)
        c = 2.0 * float((opt.w_dev * Fu).sum().item()) - float(c_energy.item())
        out = dict(rho=rho, c=c, dc=dc, lam=None, viol=0.0, P=0.0, g_rho=dc.clone())
        if opt.modal_active:
            modes, lam = self._modal()
            if self.v_ref is None:
                k = 0
            else:
                num = (modes * self.v_ref).sum(dim=(1, 2))
                a2 = (modes * modes).sum(dim=(1, 2))
                b2 = (self.v_ref * self.v_ref).sum()
                k = int(torch.argmax(num * num / torch.clamp(a2 * b2, min=1e-24)).item())
            lam1 = float(lam[k])
            v1 = modes[k]
            if self.v_ref is None:
                self.v_ref = v1.clone()
            viol = max(0.0, 1.0 - lam1 / opt.lam_t)
            qK = ctx.quadform(L.OP_K, v1[None])[0]
            qM = ctx.quadform(L.OP_M, v1[None])[0]
            vmv_tip = float((opt.tip4[:, :3] * v1[:, :3] * v1[:, :3]).sum().item())
            dlam = ctx.eig_sens(qK, qM, lam1, vmv_tip)
            out.update(lam=lam1, mode=k, dlam=dlam, viol=viol)
            if viol > 0.0:
                if self.scale is None:
                    dc_f = opt.filter.apply(dc, L.FILTER_FORWARD)
                    dl_f = opt.filter.apply(dlam, L.FILTER_FORWARD)
                    s_c = dc_f[opt.design_x].abs().mean()
                    s_m = dl_f[opt.design_x].abs().mean()
                    self.scale = float((s_c / torch.clamp(s_m, min=1e-30)).item())
                s = self.scale
                out["P"] = 0.5 * self.mu * s * opt.lam_t * viol * viol
                out["g_rho"] = dc - (self.mu * viol * s) * dlam
        out["J"] = out["c"] + out["P"]
        self.last = out
        return out

    def gradient(self, g_rho: torch.Tensor = None) -> torch.Tensor:
        """dJ/dx on the full grid (zero off the design cells)."""
        g = self.last["g_rho"] if g_rho is None else g_rho
        return self.opt.filter.apply(g, L.FILTER_ADJOINT)

    def reference_sensitivity(self) -> torch.Tensor:
        """The reference's filtered sensitivity of J (normalised filter of
        dJ/drho, src/topopt.py:311, 361), full grid."""
        return self.opt.filter.apply(self.last["g_rho"], L.FILTER_FORWARD)

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        return _ObjectiveFn.apply(x, self)


class _ObjectiveFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx_, x, objective):
        r = objective.evaluate(x)
        ctx_.objective = objective
        ctx_.g_rho = r["g_rho"]
        ctx_.in_dtype = x.dtype
        ctx_.in_device = x.device
        return torch.tensor(r["J"], dtype=torch.float64, device=x.device)

    @staticmethod
    def backward(ctx_, grad_out):
        g = ctx_.objective.gradient(ctx_.g_rho)
        g = g.to(ctx_.in_device) * grad_out.to(ctx_.in_device, torch.float64)
        return g.to(ctx_.in_dtype), None
