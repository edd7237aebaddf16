"""Oracle restatement of the SIMP optimiser (src/topopt.py) — test infrastructure.

`OracleSIMP.step()` performs one iteration of `SIMPOptimizer.run`'s loop body
(src/topopt.py:267-411) with exact FP64 solves, and returns every intermediate
the device path is compared against.
"""
from __future__ import annotations

import numpy as np
import scipy.ndimage as ndi


def cone_kernel(r_min_vox):
    """w(d) = max(0, r - d) on a (2 ceil(r) + 1)^3 box: src/topopt.py:32-41."""
    r = int(np.ceil(r_min_vox))
    c = np.arange(-r, r + 1)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    return np.maximum(0.0, r_min_vox - np.sqrt(X ** 2 + Y ** 2 + Z ** 2))


def filter_field(field_grid, mask_grid, kernel):
    """Masked normalised convolution, zero padding: src/topopt.py:44-58."""
    num = ndi.convolve(field_grid * mask_grid, kernel, mode="constant", cval=0.0)
    den = ndi.convolve(mask_grid.astype(float), kernel, mode="constant", cval=0.0)
    out = np.zeros_like(field_grid)
    out[mask_grid] = num[mask_grid] / np.maximum(den[mask_grid], 1e-12)
    return out


def filter_adjoint(grad_grid, mask_grid, kernel):
    """Exact transpose of `filter_field` as a linear map of the field on the
    mask: out_i = mask_i * sum_j w_ij mask_j g_j / den_j (the chain rule of the
    density filter; the reference itself filters sensitivities with
    `filter_field`, src/topopt.py:311)."""
    m = mask_grid.astype(float)
    den = ndi.convolve(m, kernel, mode="constant", cval=0.0)
    scaled = np.where(mask_grid, grad_grid / np.maximum(den, 1e-12), 0.0)
    # the cone kernel is symmetric, so correlation == convolution
    return ndi.convolve(scaled, kernel, mode="constant", cval=0.0) * m


def select_mode_by_mac(modes, v_prev):
    """src/topopt.py:179-188."""
    num = modes.T @ v_prev
    a2 = (modes ** 2).sum(axis=0)
    b2 = float((v_prev ** 2).sum())
    return int(np.argmax(num ** 2 / np.maximum(a2 * b2, 1e-24)))


def oc_update(x, dc, V_e, target_volume, move):
    """OC bisection on the Lagrange multiplier: src/topopt.py:190-214."""
    l1, l2 = 1e-9, 1e9
    x_new = np.empty_like(x)
    sens = np.abs(dc)
    n_bisect = 0
    while (l2 - l1) / (l1 + l2) > 1e-4:
        lmid = 0.5 * (l1 + l2)
        tmp = x * np.sqrt(sens / (lmid * V_e))
        x_new = np.maximum(0.001, np.maximum(x - move, np.minimum(1.0, np.minimum(x + move, tmp))))
        if x_new.sum() * V_e > target_volume:
            l1 = lmid
        else:
            l2 = lmid
        n_bisect += 1
    return x_new


class OracleSIMP:
    """State and loop body of `SIMPOptimizer` (src/topopt.py:64-427).

    fem: an `OracleFEM`.  F_list: full-length load vectors (one per case).
    """

    def __init__(self, geom, fem, F_list, vol_frac=0.3, r_min_mm=2.0, move=0.2,
                 weights=None, min_freq_Hz=None, tip_mass_kg=0.06, n_modes_track=4,
                 mu_freq_init=0.1, mu_freq_max=50.0, mu_freq_ramp_every=5,
                 mu_freq_ramp_factor=1.5, x0_design=None):
        self.geom, self.fem = geom, fem
        self.F_list = [np.asarray(F, float) for F in F_list]
        self.vol_frac = vol_frac
        self.r_min_vox = max(1.0, r_min_mm / (geom.dx * 1e3))       # topopt.py:109
        self.move = move
        self.min_freq_Hz = min_freq_Hz
        self.tip_mass_kg = tip_mass_kg
        self.n_modes = max(1, int(n_modes_track))
        self.mu = mu_freq_init
        self.mu_max, self.ramp_every, self.ramp_factor = mu_freq_max, max(1, int(mu_freq_ramp_every)), mu_freq_ramp_factor
        w = np.full(len(F_list), 1.0 / len(F_list)) if weights is None else np.asarray(weights, float)
        self.weights = w / w.sum()                                   # topopt.py:121-124
        m = geom.build_masks()
        self.in_arm, self.design = m["in_arm"], m["design"]
        self.active_idx = fem.elem_grid_idx
        ex, ey, ez = self.active_idx.T
        self.is_design_active = self.design[ex, ey, ez]
        self.kernel = cone_kernel(self.r_min_vox)
        self.V_e = geom.dx * geom.dy * geom.dz
        self.design_volume = int(self.is_design_active.sum()) * self.V_e
        self.target_volume = vol_frac * self.design_volume
        self.tip_nodes = (geom.motor_mount_top_nodes() if min_freq_Hz is not None
                          else np.array([], dtype=np.int64))
        # initial state: src/topopt.py:231-235 (optionally a given design start)
        rho_active = np.where(self.is_design_active, vol_frac, 1.0)
        self.rho_grid = self.to_grid(rho_active)
        if x0_design is not None:
            self.rho_grid[self.design] = np.asarray(x0_design, float)
        self.rho_phys_grid = self.rho_grid.copy()
        self.u_prev = [None] * len(F_list)
        self.v_prev = None
        self.it = 0

    def to_grid(self, vals):
        g = np.zeros((self.geom.nx, self.geom.ny, self.geom.nz))
        ex, ey, ez = self.active_idx.T
        g[ex, ey, ez] = vals
        return g

    def to_active(self, g):
        ex, ey, ez = self.active_idx.T
        return g[ex, ey, ez]

    def physical_density(self, rho_grid):
        """src/topopt.py:270-281."""
        f = filter_field(rho_grid, self.design, self.kernel)
        f[~self.design] = 0.0
        full = np.where(self.design, f, np.where(self.in_arm, 1.0, 0.0))
        return self.to_active(full)

    def step(self):
        """One loop body of src/topopt.py:267-411; returns the intermediates."""
        self.it += 1
        fem, p, emin = self.fem, self.fem.SIMP_PENALTY, self.fem.E_MIN_FRAC
        rho = self.physical_density(self.rho_grid)
        sens = np.zeros_like(self.rho_grid)
        c_total, u_list, ce_list = 0.0, [], []
        for i, F in enumerate(self.F_list):
            u, _ = fem.solve(rho, F, exact=True)
            self.u_prev[i] = u
            ce = fem.elem_compliance(u)
            c_total += self.weights[i] * float(((emin + (1 - emin) * rho ** p) * ce).sum())
            sens += self.weights[i] * self.to_grid(-p * (1 - emin) * rho ** (p - 1) * ce)
            u_list.append(u)
            ce_list.append(ce)
        sens_filt = filter_field(sens, self.design, self.kernel)
        rec = dict(rho_phys=rho, compliance=c_total, u=u_list, ce=ce_list,
                   dc_grid=sens.copy(), dc_filt=sens_filt.copy())
        if self.min_freq_Hz is not None:
            lam_t = (2 * np.pi * self.min_freq_Hz) ** 2
            freqs, modes, lam = fem.modal(rho, self.n_modes, self.tip_mass_kg, self.tip_nodes)
            k = 0 if self.v_prev is None else select_mode_by_mac(modes, self.v_prev)
            lam1, v1 = float(lam[k]), modes[:, k]
            self.v_prev = v1.copy()
            viol = max(0.0, 1.0 - lam1 / lam_t)
            rec.update(freqs=freqs, lam=lam, track_idx=k, violation=viol, mu=self.mu)
            if viol > 0.0:
                dlam = fem.eigenvalue_sensitivity(rho, lam1, v1, self.tip_mass_kg, self.tip_nodes)
                dlam_f = filter_field(self.to_grid(dlam), self.design, self.kernel)
                s_c = float(np.mean(np.abs(sens_filt[self.design])))
                s_m = float(np.mean(np.abs(dlam_f[self.design])))
                scale = s_c / max(s_m, 1e-30)
                sens_filt = sens_filt - self.mu * viol * scale * dlam_f
                rec.update(dlam=dlam, scale=scale)
            if (self.it % self.ramp_every == 0 and viol > 0.0 and self.mu < self.mu_max):
                self.mu = min(self.mu_max, self.mu * self.ramp_factor)
        x = self.rho_grid[self.design]
        x_new = oc_update(x, sens_filt[self.design], self.V_e, self.target_volume, self.move)
        new_grid = self.rho_grid.copy()
        new_grid[self.design] = x_new
        check = filter_field(new_grid, self.design, self.kernel)
        change = float(np.max(np.abs(check - self.rho_phys_grid)))
        self.rho_grid, self.rho_phys_grid = new_grid, check
        rec.update(sens_final=sens_filt, x_new=x_new, change=change,
                   vol_frac=x_new.sum() * self.V_e / self.design_volume)
        return rec
