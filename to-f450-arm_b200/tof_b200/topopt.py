"""SIMP optimiser with the reference's interface, device-resident on the B200.

Mirrors src/topopt.py: `cone_kernel`, `filter_field` and `SIMPOptimizer`
(constructor arguments, `run()` result and history keys).  One design
iteration (`step`) keeps every field on the device: density filter ->
SIMP factors -> all load cases as one block solve -> element compliances and
sensitivities -> sensitivity filter -> modal solve with MAC tracking ->
eigenvalue sensitivity and the augmented-Lagrangian frequency penalty -> OC
bisection -> change; only scalars (compliance, eigenvalues, change) reach the
host, as the reference's control flow needs them.
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

from . import _lib as L
from .engine import DensityFilter, oc_update


def cone_kernel(r_min_vox: float) -> np.ndarray:
    """w(d) = max(0, r - d) on a (2 ceil(r) + 1)^3 box (src/topopt.py:32-41)."""
    r = int(np.ceil(r_min_vox))
    c = np.arange(-r, r + 1)
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    return np.maximum(0.0, r_min_vox - np.sqrt(X ** 2 + Y ** 2 + Z ** 2))


def _grid_to_dev(a, device):
    """(nx, ny, nz) array -> device FP64 (NE,), x fastest."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float64).transpose(2, 1, 0).ravel())).to(device)


def _dev_to_grid(t, shape):
    nx, ny, nz = shape
    return t.reshape(nz, ny, nx).permute(2, 1, 0).cpu().numpy().copy()


_filters = {}


def filter_field(field_grid: np.ndarray, mask_grid: np.ndarray, kernel: np.ndarray) -> np.ndarray:
    """Masked normalised convolution (src/topopt.py:44-58), on the GPU."""
    shape = np.shape(field_grid)
    key = (shape, np.asarray(mask_grid, bool).tobytes(), np.asarray(kernel, float).tobytes())
    f = _filters.get(key)
    if f is None:
        f = _filters[key] = DensityFilter(shape, kernel, mask_grid)
    dev = torch.device("cuda", torch.cuda.current_device())
    out = f.apply(_grid_to_dev(field_grid, dev))
    return _dev_to_grid(out, shape)


class SIMPOptimizer:
    """Run SIMP topology optimisation (src/topopt.py:64-427) on the device.

    Extra keyword arguments (not in the reference):
      batch_loads  - solve all load cases as one block (default True);
      concurrent   - in the mixed form, run the static solves and the modal
                     solve of an iteration at the same time on two CUDA
                     streams from two host threads (default True; each is a
                     chain of short, latency-bound kernels that leaves most of
                     the GPU idle, and the library keeps separate scratch for
                     the two);
      solve_rtol   - static solve tolerance (default fem.SOLVE_RTOL);
      modal_tol    - LOBPCG relative residual tolerance (default 1e-5);
      x0_design    - start values on the design cells (reference order);
      modal_maxiter - LOBPCG iteration cap (default 20000 Jacobi / 1000 multigrid);
      F_list       - explicit full-length load vectors instead of load_cases.
    """

    def __init__(self, geom, fem, load_cases: list, vol_frac: float = 0.30, r_min_mm: float = 2.0,
                 move: float = 0.2, max_iter: int = 100, tol_change: float = 0.01, weights: list = None,
                 min_freq_Hz: float = None, tip_mass_kg: float = 0.060, n_modes_track: int = 4,
                 mu_freq_init: float = 0.10, mu_freq_max: float = 50.0, mu_freq_ramp_every: int = 5,
                 mu_freq_ramp_factor: float = 1.5, batch_loads: bool = True, solve_rtol: float = None,
                 modal_tol: float = 1e-5, x0_design=None, F_list=None, modal_maxiter: int = None,
                 concurrent: bool = True):
        self.geom, self.fem = geom, fem
        self.load_cases = load_cases
        self.vol_frac = vol_frac
        self.r_min_vox = max(1.0, r_min_mm / (geom.dx * 1e3))               # src/topopt.py:109
        self.move, self.max_iter, self.tol_change = move, max_iter, tol_change
        self.min_freq_Hz, self.tip_mass_kg = min_freq_Hz, tip_mass_kg
        self.n_modes_track = max(1, int(n_modes_track))
        self.mu_freq, self.mu_freq_max = mu_freq_init, mu_freq_max
        self.mu_freq_ramp_every = max(1, int(mu_freq_ramp_every))
        self.mu_freq_ramp_factor = mu_freq_ramp_factor
        self.batch_loads = batch_loads
        self.concurrent = concurrent
        self._side = None                     # (static, modal) streams of the concurrent step
        self._worker = None                   # the host thread that issues the static solves
        self.solve_rtol = fem.SOLVE_RTOL if solve_rtol is None else solve_rtol
        self.modal_tol = modal_tol
        self.modal_maxiter = modal_maxiter
        self.modal_mg_cycles = 1              # V-cycles per LOBPCG preconditioner application
        n_lc = len(F_list) if F_list is not None else len(load_cases)
        w = np.full(n_lc, 1.0 / n_lc) if weights is None else np.asarray(weights, dtype=float)
        self.weights = w / w.sum()                                           # src/topopt.py:121-124
        m = geom.build_masks()
        self.in_arm, self.design, self.keep_solid = m["in_arm"], m["design"], m["keep_solid"]
        self.active_idx = fem.elem_grid_idx
        ex, ey, ez = self.active_idx.T
        self.is_design_active = self.design[ex, ey, ez]
        self.n_design = int(self.is_design_active.sum())
        self.kernel = cone_kernel(self.r_min_vox)
        self.design_mask_grid = self.design.astype(bool)
        if F_list is None:                                                   # src/topopt.py:148-158
            F_list = []
            for lc in load_cases:
                F = np.zeros(geom.n_dofs)
                if lc.get("F") is not None:
                    d, v = geom.load_dofs_for_force(lc["F"])
                    np.add.at(F, d, v)
                if lc.get("Mz") is not None:
                    d, v = geom.load_dofs_for_moment_Mz(lc["Mz"])
                    np.add.at(F, d, v)
                F_list.append(F)
        self.F_list = [np.asarray(F, dtype=np.float64) for F in F_list]
        self.V_e = geom.dx * geom.dy * geom.dz
        self.design_volume = self.n_design * self.V_e
        self.target_volume = vol_frac * self.design_volume
        self._x0_design = None if x0_design is None else np.asarray(x0_design, dtype=np.float64)
        self._setup_device()

    # ------------------------------------------------------------------ #
    def _setup_device(self):
        fem, geom = self.fem, self.geom
        self.ctx = ctx = fem.device()
        dev = ctx.device
        self.dev = dev
        shape = (geom.nx, geom.ny, geom.nz)
        self.shape = shape
        design_x = np.asarray(self.design, bool).transpose(2, 1, 0).ravel()
        arm_x = np.asarray(self.in_arm, bool).transpose(2, 1, 0).ravel()
        # design cells in the reference's order (grid[design] on the (nx,ny,nz) C-order array)
        gx, gy, gz = np.nonzero(self.design)
        self.design_ids = torch.as_tensor(gz * geom.nx * geom.ny + gy * geom.nx + gx, device=dev)
        self.design_x = torch.as_tensor(design_x, device=dev)
        self.filter = DensityFilter(shape, self.kernel, self.design, fill_grid=self.in_arm & ~self.design)
        self.b4 = ctx.pack(torch.from_numpy(np.stack(self.F_list)))
        self.w_dev = torch.as_tensor(self.weights, dtype=torch.float64, device=dev)
        self.modal_active = self.min_freq_Hz is not None
        self.tip_nodes = fem._tip_nodes(None) if self.modal_active else np.array([], dtype=np.int64)
        tip = fem.tip_lump(self.tip_mass_kg, self.tip_nodes) if self.modal_active else None
        self._tip3 = tip
        self._tip_key = None if tip is None else tip.tobytes()
        self.tip4 = ctx.pack(torch.from_numpy(np.zeros(geom.n_dofs) if tip is None else tip))[0]
        self.profile = False          # True: synchronised per-phase timings in self.phase_times
        self.phase_times = {}
        self.lam_t = (2.0 * np.pi * self.min_freq_Hz) ** 2 if self.modal_active else None
        self.reset()

    def set_loads(self, F_list):
        """Replace the load vectors (same count as the weights)."""
        if len(F_list) != len(self.weights):
            raise ValueError("number of load vectors must match the weights")
        self.F_list = [np.asarray(F, dtype=np.float64) for F in F_list]
        self.b4 = self.ctx.pack(torch.from_numpy(np.stack(self.F_list)))

    def reset(self):
        """Initial state of src/topopt.py:231-257."""
        ctx = self.ctx
        x = torch.zeros(ctx.NE, dtype=torch.float64, device=self.dev)
        arm_x = torch.as_tensor(np.asarray(self.in_arm, bool).transpose(2, 1, 0).ravel(), device=self.dev)
        x[arm_x] = 1.0
        x[self.design_x] = self.vol_frac
        if self._x0_design is not None:
            x[self.design_ids] = torch.as_tensor(self._x0_design, device=self.dev)
        self.x = x
        self.rho_phys_prev = x.clone()          # the reference compares against this first
        self.u4 = None
        self.X4 = None
        self.v_prev = None
        self.it = 0
        self.mu_freq_cur = self.mu_freq
        self.history = {"compliance": [], "mass": [], "change": [], "vol_frac": [], "omega_1_Hz": [],
                        "mu_freq": [], "freq_violation": [], "modal_converged": [], "modal_iters": [],
                        "modal_relres": [], "pcg_iters": [], "pcg_relres": []}
        self.stats = []

    # ------------------------------------------------------------------ #
    def _mark(self, name):
        """Phase timer (only when self.profile is set; synchronises)."""
        if not self.profile:
            return
        torch.cuda.synchronize()
        now = time.perf_counter()
        if name is not None:
            self.phase_times[name] = self.phase_times.get(name, 0.0) + now - self._t_mark
        self._t_mark = now

    def physical_density(self, x=None) -> torch.Tensor:
        """Filtered design, keep-solid = 1, inactive = 0 (src/topopt.py:270-281)."""
        return self.filter.apply(self.x if x is None else x, L.FILTER_PHYSICAL)

    def _modal(self, rho_grid):
        fem, ctx = self.fem, self.ctx
        n = self.n_modes_track
        nb = min(fem.max_modes, n + 2)
        if self.X4 is None:                                  # src/fem.py:448-449 start block
            n_free = len(fem.free_dofs)
            X0 = np.random.default_rng(0).standard_normal((n_free, n))
            extra = np.random.default_rng(1).standard_normal((n_free, nb - n))
            full = np.zeros((nb, self.geom.n_dofs))
            full[:, fem.free_dofs] = np.concatenate([X0, extra], axis=1).T
            X4 = ctx.pack(torch.from_numpy(full))
        else:
            X4 = self.X4
        mid = fem._mode_id()
        maxit = self.modal_maxiter or (20000 if mid == L.MODE_FP64 else 1000)
        modes, lam, st = ctx.lobpcg(X4, n, tol=self.modal_tol, maxiter=maxit, mode=mid,
                                    precond=L.PRECOND_MG if mid == L.MODE_MIXED else L.PRECOND_JACOBI,
                                    mg_cycles=self.modal_mg_cycles)
        # warm start: the final Ritz vectors, modes and guard vectors
        self.X4 = ctx.last_block
        self.stats.append(("lobpcg", st))
        self.history["modal_converged"].append(st["status"] == L.TOF_OK)
        self.history["modal_iters"].append(st["iters"])
        self.history["modal_relres"].append(st["relres"])
        return modes, np.maximum(lam, 0.0)

    def _static(self, mid):
        """All load cases as one block (src/topopt.py:287-306), then the
        weighted compliance and its filtered sensitivity (src/topopt.py:307-311).
        Returns (filtered sensitivity, compliance as a device scalar)."""
        ctx = self.ctx
        R = self.b4.shape[0]
        if self.batch_loads and mid == L.MODE_MIXED:
            u4, st = ctx.pcg(self.b4, self.u4, rtol=self.solve_rtol, maxiter=20000, mode=mid)
        else:
            parts, st = [], []
            for i in range(R):
                ui, si = ctx.pcg(self.b4[i:i + 1], None if self.u4 is None else self.u4[i:i + 1],
                                 rtol=self.solve_rtol, maxiter=20000, mode=mid)
                parts.append(ui)
                st += si
            u4 = torch.cat(parts)
        self.u4 = u4
        self.stats.append(("pcg", st))
        self.history["pcg_iters"].append(max(s["iters"] for s in st))
        self.history["pcg_relres"].append(max(s["relres"] for s in st))
        ce = ctx.quadform(L.OP_K, u4)
        c_dev, dc = ctx.compliance_sens(ce, self.w_dev)
        sens = self.filter.apply(dc, L.FILTER_FORWARD)       # src/topopt.py:311
        return sens, c_dev

    def step(self):
        """One iteration of src/topopt.py:267-411; returns the change."""
        self.it += 1
        it = self.it
        t0 = time.time()
        fem, ctx = self.fem, self.ctx
        p, emin = fem.SIMP_PENALTY, fem.E_MIN_FRAC
        self._mark(None)
        rho = self.physical_density()
        ctx.set_density(rho)
        fem._rho_dev = None                                  # the FEM3D cache no longer matches
        if self.modal_active and (fem._tip_key is None or fem._tip_key != self._tip_key):
            ctx.set_tip_lump(self._tip3)
            fem._tip_key = self._tip_key
        self._mark("filter+density")
        # --- all load cases (src/topopt.py:287-306) and the modes
        # (src/topopt.py:313-330): independent given the density
        mid = fem._mode_id()
        if self.concurrent and self.modal_active and mid == L.MODE_MIXED:
            ctx.mg_setup()                                    # on the stream both sides wait on
            main = torch.cuda.current_stream()
            if self._side is None:
                self._side = (torch.cuda.Stream(device=self.dev), torch.cuda.Stream(device=self.dev))
                self._worker = ThreadPoolExecutor(max_workers=1, thread_name_prefix="tof-static")
            s_static, s_modal = self._side
            s_static.wait_stream(main)
            s_modal.wait_stream(main)

            def static_side():
                # the worker waits for its own stream (free: the static side
                # ends well before the modal side on these designs)
                with torch.cuda.stream(s_static):
                    out = self._static(mid)
                s_static.synchronize()
                return out

            fut = self._worker.submit(static_side)
            modal_exc = None
            try:
                with torch.cuda.stream(s_modal):
                    modes, lam = self._modal(rho)
            except BaseException as e:                        # raised after the static side joined
                modal_exc = e
            static_exc = fut.exception()
            main.wait_stream(s_static)
            main.wait_stream(s_modal)
            if modal_exc is not None:
                raise modal_exc
            if static_exc is not None:
                raise static_exc
            sens, c_dev = fut.result()
            self._mark("static + modal solves")
        else:
            sens, c_dev = self._static(mid)
            self._mark("static solves")
            if self.modal_active:
                modes, lam = self._modal(rho)
                self._mark("modal solve")
        c_total = float(c_dev.item())
        # --- modal constraint (src/topopt.py:313-375)
        if self.modal_active:
            if self.v_prev is None:
                k = 0
            else:                                            # MAC, src/topopt.py:179-188
                num = (modes * self.v_prev).sum(dim=(1, 2))
                a2 = (modes * modes).sum(dim=(1, 2))
                b2 = (self.v_prev * self.v_prev).sum()
                mac = num * num / torch.clamp(a2 * b2, min=1e-24)
                k = int(torch.argmax(mac).item())
            lam1 = float(lam[k])
            v1 = modes[k]
            self.v_prev = v1.clone()
            viol = max(0.0, 1.0 - lam1 / self.lam_t)
            if viol > 0.0:
                qK = ctx.quadform(L.OP_K, v1[None])[0]
                qM = ctx.quadform(L.OP_M, v1[None])[0]
                vmv_tip = float((self.tip4[:, :3] * v1[:, :3] * v1[:, :3]).sum().item())
                dlam = ctx.eig_sens(qK, qM, lam1, vmv_tip)
                dlam_f = self.filter.apply(dlam, L.FILTER_FORWARD)
                s_c = sens[self.design_x].abs().mean()
                s_m = dlam_f[self.design_x].abs().mean()
                scale = s_c / torch.clamp(s_m, min=1e-30)
                sens = sens - (self.mu_freq_cur * viol) * scale * dlam_f
            self.history["omega_1_Hz"].append(float(np.sqrt(lam1) / (2 * np.pi)))
            self.history["mu_freq"].append(self.mu_freq_cur)
            self.history["freq_violation"].append(viol)
            if (it % self.mu_freq_ramp_every == 0 and viol > 0.0 and self.mu_freq_cur < self.mu_freq_max):
                self.mu_freq_cur = min(self.mu_freq_max, self.mu_freq_cur * self.mu_freq_ramp_factor)
        else:
            for k in ("omega_1_Hz", "mu_freq", "freq_violation"):
                self.history[k].append(np.nan)
        self._mark("eigen sens+penalty")
        # --- OC on design cells (src/topopt.py:377-390)
        self.last_sensitivity = sens                         # what OC receives (full grid)
        x_d = self.x[self.design_ids]
        x_new_d = oc_update(x_d, sens[self.design_ids], self.V_e, self.target_volume, self.move)
        x_new = self.x.clone()
        x_new[self.design_ids] = x_new_d
        check = self.filter.apply(x_new, L.FILTER_FORWARD)
        change = float((check - self.rho_phys_prev).abs().max().item())
        self.x, self.rho_phys_prev = x_new, check
        mass = float(x_new_d.sum().item()) * self.V_e
        self.history["compliance"].append(c_total)
        self.history["mass"].append(mass)
        self.history["change"].append(change)
        self.history["vol_frac"].append(mass / self.design_volume)
        self._mark("OC+change")
        self.last_step_s = time.time() - t0
        return change

    def run(self, verbose: bool = True):
        """src/topopt.py:217-427; returns rho_active, rho_grid, history, u_per_lc."""
        if verbose:
            print(f"SIMP TO start (B200) - target Vf = {self.vol_frac:.3f}, r_min = {self.r_min_vox:.2f} vox")
        for it in range(1, self.max_iter + 1):
            change = self.step()
            if verbose:
                h = self.history
                extra = ""
                if self.modal_active:
                    extra = f"  w1={h['omega_1_Hz'][-1]:6.1f}Hz  mu={self.mu_freq_cur:.2e}"
                print(f"  iter {it:3d}  c={h['compliance'][-1]:.4e}  Vf={h['vol_frac'][-1]:.3f}  "
                      f"change={change:.4f}  [{self.last_step_s:.3f}s]{extra}")
            if change < self.tol_change and it > 10:
                break
        rho = self.physical_density()
        rho_grid = _dev_to_grid(rho, self.shape)
        rho_active = rho[torch.as_tensor(self.fem.active_ids, device=self.dev)].cpu().numpy()
        u = self.ctx.unpack(self.u4).cpu().numpy() if self.u4 is not None else None
        return {"rho_active": rho_active, "rho_grid": rho_grid, "history": self.history,
                "u_per_lc": None if u is None else [u[i] for i in range(u.shape[0])]}
