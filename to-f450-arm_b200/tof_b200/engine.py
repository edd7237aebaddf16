"""Device-resident design context: the Python face of one libtof context.

Holds the libtof handle for one voxel design plus the torch device buffers
that cross the C ABI.  All arrays here are torch CUDA tensors in the library's
layouts (node4 vectors (R, NN, 4); element grids (NE,) x fastest); the
reference-shaped NumPy API lives in `tof_b200.fem`.  Every call runs on
torch's current CUDA stream, so library kernels and torch ops stay ordered.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_uint8, c_void_p

import numpy as np
import torch

from . import _lib as L


def _stream():
    return c_void_p(torch.cuda.current_stream().cuda_stream)


class DesignContext:
    """One structured-grid design on the current CUDA device."""

    def __init__(self, nx, ny, nz, h, Ke, Me, active_grid=None, fixed_dofs=(), tip_lump=None,
                 simp=(3.0, 1e-9, 0.1, 6.0), max_rhs=8, max_modes=8, tile=None):
        if not torch.cuda.is_available():
            raise RuntimeError("tof_b200 needs a CUDA device (no CPU fallback)")
        self.lib = L.load()
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.NX, self.NY, self.NZ = self.nx + 1, self.ny + 1, self.nz + 1
        self.NN = self.NX * self.NY * self.NZ
        self.NE = self.nx * self.ny * self.nz
        self.N = 3 * self.NN
        self.device = torch.device("cuda", torch.cuda.current_device())
        Ke = np.ascontiguousarray(Ke, dtype=np.float64).reshape(576)
        Me = np.ascontiguousarray(Me, dtype=np.float64).reshape(576)
        if active_grid is None:
            act = np.ones(self.NE, np.uint8)
        else:
            act = np.ascontiguousarray(np.asarray(active_grid, bool).transpose(2, 1, 0).ravel(), np.uint8)
        fixed = np.zeros(self.N, np.uint8)
        fixed[np.asarray(fixed_dofs, dtype=np.int64)] = 1
        tip = None if tip_lump is None else np.ascontiguousarray(tip_lump, np.float64)
        sp = L.SimpParams(*simp)
        h3 = np.ascontiguousarray(h, np.float64)
        tl = None if tile is None else (c_int * 3)(*tile)
        handle = c_void_p()
        rc = self.lib.tof_ctx_create(self.nx, self.ny, self.nz, L.dptr(h3), L.dptr(Ke), L.dptr(Me),
                                     act.ctypes.data_as(POINTER(c_uint8)),
                                     fixed.ctypes.data_as(POINTER(c_uint8)),
                                     None if tip is None else L.dptr(tip), ctypes.byref(sp),
                                     int(max_rhs), int(max_modes), tl, ctypes.byref(handle))
        L.check("tof_ctx_create", rc)
        self.h = handle
        self.max_rhs = int(self.lib.tof_ctx_query(self.h, L.Q_MAX_RHS))
        self.max_modes = int(self.lib.tof_ctx_query(self.h, L.Q_MAX_MODES))
        self.n_free = int(self.lib.tof_ctx_query(self.h, L.Q_FREE_DOFS))
        self.tile = tuple(int(self.lib.tof_ctx_query(self.h, q)) for q in (L.Q_TILE_X, L.Q_TILE_Y, L.Q_TILE_Z))
        self.active = torch.from_numpy(act.astype(bool)).to(self.device)
        self.last_stats = []
        self.last_rc = None

    def close(self):
        if getattr(self, "h", None):
            torch.cuda.synchronize()
            self.lib.tof_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ #
    def zeros4(self, R, dtype=torch.float64):
        return torch.zeros((R, self.NN, 4), dtype=dtype, device=self.device)

    def set_density(self, rho_grid: torch.Tensor):
        """rho over the full element grid (NE,), FP64, x fastest."""
        rho_grid = rho_grid.to(self.device, torch.float64).contiguous()
        L.check("tof_set_density", self.lib.tof_set_density(self.h, L.ptr(rho_grid), _stream()), self.h)
        self._rho_keep = rho_grid

    def set_tip_lump(self, tip3):
        t = None if tip3 is None else np.ascontiguousarray(tip3, np.float64)
        L.check("tof_set_tip_lump", self.lib.tof_set_tip_lump(self.h, None if t is None else L.dptr(t),
                                                              _stream()), self.h)

    def pack(self, dofs: torch.Tensor, dtype=torch.float64) -> torch.Tensor:
        """(R, 3NN) or (3NN,) FP64 DOF-major -> node4 (R, NN, 4), zero at fixed DOFs."""
        d = dofs.to(self.device, torch.float64)
        if d.dim() == 1:
            d = d[None]
        d = d.contiguous()
        out = torch.empty((d.shape[0], self.NN, 4), dtype=dtype, device=self.device)
        L.check("tof_pack", self.lib.tof_pack(self.h, L.ptr(d), d.shape[1], L.ptr(out),
                                              L.F64 if dtype == torch.float64 else L.F32, d.shape[0],
                                              _stream()), self.h)
        return out

    def unpack(self, v4: torch.Tensor) -> torch.Tensor:
        """node4 (R, NN, 4) -> (R, 3NN) FP64."""
        v4 = v4.contiguous()
        out = torch.empty((v4.shape[0], self.N), dtype=torch.float64, device=self.device)
        L.check("tof_unpack", self.lib.tof_unpack(self.h, L.ptr(v4), L.F64 if v4.dtype == torch.float64 else L.F32,
                                                  L.ptr(out), self.N, v4.shape[0], _stream()), self.h)
        return out

    def matvec(self, op: int, x4: torch.Tensor) -> torch.Tensor:
        x4 = x4.contiguous()
        y = torch.empty_like(x4)
        L.check("tof_matvec", self.lib.tof_matvec(self.h, op, L.F64 if x4.dtype == torch.float64 else L.F32,
                                                  L.ptr(x4), L.ptr(y), x4.shape[0], _stream()), self.h)
        return y

    def diag(self, op: int) -> torch.Tensor:
        out = self.zeros4(1)[0]
        L.check("tof_diag", self.lib.tof_diag(self.h, op, L.ptr(out), _stream()), self.h)
        return out

    def pcg(self, b4: torch.Tensor, x4: torch.Tensor = None, rtol=1e-8, maxiter=20000, mode=L.MODE_MIXED,
            raise_on_error=True):
        """Solve K x = b for R node4 FP64 rhs; returns (x4, stats list)."""
        b4 = b4.contiguous()
        R = b4.shape[0]
        x = self.zeros4(R) if x4 is None else x4.to(torch.float64).contiguous().clone()
        st = (L.SolveStats * R)()
        rc = self.lib.tof_pcg(self.h, mode, L.ptr(b4), L.ptr(x), R, float(rtol), int(maxiter), st, _stream())
        stats = [dict(status=s.status, iters=s.iters, outer=s.outer, relres=s.relres, floor=s.floor) for s in st]
        self.last_stats = stats
        self.last_rc = rc
        if raise_on_error:
            L.check("tof_pcg", rc, self.h, allow=(L.TOF_OK, L.TOF_NOT_CONVERGED))
        return x, stats

    def lobpcg(self, X4: torch.Tensor, nmodes: int, tol=1e-5, maxiter=500, mode=L.MODE_MIXED,
               precond=L.PRECOND_PCG, inner_iters=60, inner_rtol=1e-2, raise_on_error=True, mg_cycles=1):
        """Lowest nmodes of K x = lam M x from the start block X4 (block, NN, 4).
        mg_cycles: V-cycles per preconditioner application (multigrid).
        Returns the modes (the first nmodes Ritz vectors); all `block` Ritz
        vectors of the final step are kept in self.last_block."""
        if precond == L.PRECOND_MG or mode == L.MODE_MIXED:
            inner_iters = mg_cycles
        X = X4.to(torch.float64).contiguous().clone()
        block = X.shape[0]
        lam = (c_double * nmodes)()
        res = (c_double * nmodes)()
        st = L.SolveStats()
        rc = self.lib.tof_lobpcg(self.h, mode, nmodes, block, L.ptr(X), lam, float(tol), int(maxiter), precond,
                                 int(inner_iters), float(inner_rtol), ctypes.byref(st), res, _stream())
        stats = dict(status=st.status, iters=st.iters, relres=st.relres, floor=st.floor, resid=list(res))
        self.last_stats = [stats]
        self.last_rc = rc
        self.last_block = X
        if raise_on_error:
            L.check("tof_lobpcg", rc, self.h, allow=(L.TOF_OK, L.TOF_NOT_CONVERGED))
        return X[:nmodes], np.array(list(lam)), stats

    def quadform(self, op: int, v4: torch.Tensor) -> torch.Tensor:
        """(R, NE) FP64 per-element v_e^T A_e v_e."""
        v4 = v4.contiguous()
        out = torch.empty((v4.shape[0], self.NE), dtype=torch.float64, device=self.device)
        L.check("tof_elem_quadform", self.lib.tof_elem_quadform(
            self.h, op, L.F64 if v4.dtype == torch.float64 else L.F32, L.ptr(v4), v4.shape[0], L.ptr(out),
            _stream()), self.h)
        return out

    def gram(self, A4, B4) -> torch.Tensor:
        G = torch.empty((A4.shape[0], B4.shape[0]), dtype=torch.float64, device=self.device)
        L.check("tof_gram", self.lib.tof_gram(self.h, L.F64 if A4.dtype == torch.float64 else L.F32, L.ptr(A4),
                                              A4.shape[0], L.ptr(B4), B4.shape[0], L.ptr(G), _stream()), self.h)
        return G

    def compliance_sens(self, ce: torch.Tensor, weights: torch.Tensor):
        """(c scalar tensor, dc (NE,)) from ce (nlc, NE) at the current density."""
        ce = ce.contiguous()
        w = weights.to(self.device, torch.float64).contiguous()
        dc = torch.empty(self.NE, dtype=torch.float64, device=self.device)
        c = torch.empty(1, dtype=torch.float64, device=self.device)
        L.check("tof_compliance_sens", self.lib.tof_compliance_sens(self.h, ce.shape[0], L.ptr(w), L.ptr(ce),
                                                                    L.ptr(dc), L.ptr(c), _stream()), self.h)
        return c, dc

    def eig_sens(self, qK: torch.Tensor, qM: torch.Tensor, lam: float, vMv_tip: float) -> torch.Tensor:
        out = torch.empty(self.NE, dtype=torch.float64, device=self.device)
        L.check("tof_eig_sens", self.lib.tof_eig_sens(self.h, L.ptr(qK.contiguous()), L.ptr(qM.contiguous()),
                                                      float(lam), float(vMv_tip), L.ptr(out), _stream()), self.h)
        return out

    # -- multigrid introspection ------------------------------------------ #
    def mg_levels(self):
        """[(nx, ny, nz, omega)] per multigrid level (omega 0 on the coarsest)."""
        n = self.lib.tof_mg_query(self.h, -1, None, None, _stream())
        out = []
        for lv in range(n):
            dims = (c_int * 3)()
            om = ctypes.c_float()
            L.check("tof_mg_query", min(0, self.lib.tof_mg_query(self.h, lv, dims, ctypes.byref(om), _stream())),
                    self.h)
            out.append((dims[0], dims[1], dims[2], om.value))
        return out

    def mg_element_matrices(self, level: int) -> torch.Tensor:
        nx, ny, nz, _ = self.mg_levels()[level]
        out = torch.empty((nx * ny * nz, 24, 24), dtype=torch.float32, device=self.device)
        L.check("tof_mg_export", self.lib.tof_mg_export(self.h, level, L.ptr(out), _stream()), self.h)
        return out

    def mg_setup(self):
        """Build the multigrid hierarchy for the current density now, on the
        current stream (before a static and a modal solve run concurrently)."""
        L.check("tof_mg_setup", self.lib.tof_mg_setup(self.h, _stream()), self.h)

    def mg_apply(self, r4: torch.Tensor) -> torch.Tensor:
        r4 = r4.to(torch.float32).contiguous()
        e = torch.empty_like(r4)
        L.check("tof_mg_apply", self.lib.tof_mg_apply(self.h, L.ptr(r4), L.ptr(e), r4.shape[0], _stream()), self.h)
        return e

    def stress(self, u4: torch.Tensor, B_c: np.ndarray, D: np.ndarray, rho_grid: torch.Tensor = None,
               sigma=True, vm=True, smax=True):
        """Element-centre stress of R node4 displacement vectors over the full
        grid: (sigma (R, NE, 6), vm (R, NE), smax (R, NE)), each None unless
        requested.  rho_grid None: the density set by set_density."""
        u4 = u4.contiguous()
        R = u4.shape[0]
        dev = self.device
        o_s = torch.empty((R, self.NE, 6), dtype=torch.float64, device=dev) if sigma else None
        o_v = torch.empty((R, self.NE), dtype=torch.float64, device=dev) if vm else None
        o_m = torch.empty((R, self.NE), dtype=torch.float64, device=dev) if smax else None
        rho = None if rho_grid is None else rho_grid.to(dev, torch.float64).contiguous()
        Bc = np.ascontiguousarray(B_c, np.float64)
        Dm = np.ascontiguousarray(D, np.float64)
        L.check("tof_stress", self.lib.tof_stress(self.h, L.dptr(Bc), L.dptr(Dm),
                                                  L.F64 if u4.dtype == torch.float64 else L.F32, L.ptr(u4), R,
                                                  L.ptr(rho), L.ptr(o_s), L.ptr(o_v), L.ptr(o_m), _stream()), self.h)
        return o_s, o_v, o_m

    def effective_mass(self, modes4: torch.Tensor, direction=2) -> np.ndarray:
        m = modes4.to(torch.float64).contiguous()
        out = (c_double * m.shape[0])()
        L.check("tof_effective_mass", self.lib.tof_effective_mass(self.h, L.ptr(m), m.shape[0], int(direction),
                                                                  out, _stream()), self.h)
        return np.array(list(out))


class DensityFilter:
    """libtof density filter on an (nx, ny, nz) element grid (x fastest on device)."""

    def __init__(self, shape, weights: np.ndarray, mask_grid: np.ndarray, fill_grid: np.ndarray = None):
        self.lib = L.load()
        nx, ny, nz = shape
        self.shape = (nx, ny, nz)
        w = np.asarray(weights, np.float64)
        kx, ky, kz = w.shape
        # the kernel array is indexed [qx, qy, qz]; the C ABI wants z slowest
        wz = np.ascontiguousarray(w.transpose(2, 1, 0))
        m = np.ascontiguousarray(np.asarray(mask_grid, bool).transpose(2, 1, 0).ravel(), np.uint8)
        f = None if fill_grid is None else np.ascontiguousarray(
            np.asarray(fill_grid, bool).transpose(2, 1, 0).ravel(), np.uint8)
        h = c_void_p()
        rc = self.lib.tof_filter_create(nx, ny, nz, L.dptr(wz), kx, ky, kz, m.ctypes.data_as(POINTER(c_uint8)),
                                        None if f is None else f.ctypes.data_as(POINTER(c_uint8)), ctypes.byref(h))
        L.check("tof_filter_create", rc)
        self.h = h

    def apply(self, x: torch.Tensor, mode=L.FILTER_FORWARD) -> torch.Tensor:
        x = x.to(torch.float64).contiguous()
        out = torch.empty_like(x)
        L.check("tof_filter_apply", self.lib.tof_filter_apply(self.h, mode, L.ptr(x), L.ptr(out), _stream()))
        return out

    def __del__(self):
        try:
            if self.h:
                self.lib.tof_filter_destroy(self.h)
                self.h = None
        except Exception:
            pass


def stress_invariants(sigma: torch.Tensor):
    """(von Mises, largest principal stress) of (..., 6) Voigt stresses on the
    device (src/fem.py:582-602)."""
    lib = L.load()
    s = sigma.to(torch.float64).contiguous()
    n = s.numel() // 6
    vm = torch.empty(s.shape[:-1], dtype=torch.float64, device=s.device)
    smax = torch.empty_like(vm)
    L.check("tof_stress_invariants", lib.tof_stress_invariants(n, L.ptr(s), L.ptr(vm), L.ptr(smax), _stream()))
    return vm, smax


def oc_update(x: torch.Tensor, dc: torch.Tensor, V_e: float, target_volume: float, move: float) -> torch.Tensor:
    lib = L.load()
    x = x.to(torch.float64).contiguous()
    dc = dc.to(torch.float64).contiguous()
    out = torch.empty_like(x)
    L.check("tof_oc_update", lib.tof_oc_update(x.numel(), L.ptr(x), L.ptr(dc), float(V_e), float(target_volume),
                                               float(move), L.ptr(out), None, _stream()))
    return out
