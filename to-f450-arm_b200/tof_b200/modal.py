"""Modal effective mass in the thrust direction (sims/modal_participation.py).

`effective_mass_voxel` has the reference's signature
(sims/modal_participation.py:37) and computes
(phi^T M r)^2 / (phi^T M phi) / (r^T M r) with the same consistent mass and
tip lump the eigensolve used, on the device (one block M product and one Gram
matrix).
"""
from __future__ import annotations

import numpy as np
import torch

EXCITABLE_FRAC = 0.05          # sims/modal_participation.py:34


def effective_mass_voxel(fem, geom, rho_active, mode_shapes, tip_mass_kg, direction=2):
    """Effective-mass fraction per mode (sims/modal_participation.py:37-57).
    `fem` is a tof_b200.fem.FEM3D; mode_shapes is (N, m)."""
    nodes = geom.motor_mount_top_nodes()
    ctx = fem._prepare(rho_active, tip_mass_kg, nodes)
    modes = np.asarray(mode_shapes, dtype=np.float64)
    m4 = ctx.pack(torch.from_numpy(np.ascontiguousarray(modes.T)))
    return ctx.effective_mass(m4, direction)


def first_excitable(freqs, eff, thresh=EXCITABLE_FRAC):
    """(frequency, effective-mass fraction, index) of the lowest excitable mode
    (sims/modal_participation.py:89-94)."""
    for k, (f, e) in enumerate(zip(freqs, eff)):
        if e >= thresh:
            return float(f), float(e), k
    return None, None, None


def rank_by_effective_mass(freqs, eff):
    """Mode indices ordered by effective mass, largest first."""
    return list(np.argsort(-np.asarray(eff), kind="stable"))


def modal_frf(freqs_Hz, V, f_Hz, modal_damping=0.02):
    """|H_dd(f)| at several DOFs on the device: V (ndof, m) mode-shape values
    at the DOFs (numpy or a CUDA tensor), f_Hz the frequency grid.  Returns a
    (ndof, len(f_Hz)) CUDA tensor (src/plotting.py:378-399, batched)."""
    from . import _lib as L
    from .engine import _stream
    dev = torch.device("cuda", torch.cuda.current_device())
    Vt = torch.as_tensor(V, dtype=torch.float64, device=dev)
    if Vt.dim() == 1:
        Vt = Vt[None]
    Vt = Vt.contiguous()
    fk = torch.as_tensor(np.asarray(freqs_Hz, dtype=np.float64), device=dev).contiguous()
    f = torch.as_tensor(np.asarray(f_Hz, dtype=np.float64), device=dev).contiguous()
    out = torch.empty((Vt.shape[0], f.numel()), dtype=torch.float64, device=dev)
    L.check("tof_modal_frf", L.load().tof_modal_frf(Vt.shape[0], Vt.shape[1], L.ptr(Vt), L.ptr(fk), f.numel(),
                                                   L.ptr(f), float(modal_damping), L.ptr(out), _stream()))
    return out


def modal_frf_at_dof(frequencies_Hz, mode_shapes, dof_idx: int, freq_range_Hz: tuple = (10.0, 1500.0),
                     n_pts: int = 600, modal_damping: float = 0.02) -> tuple:
    """(freqs_Hz, |H|) of the modal-superposition FRF at one DOF with the
    reference's signature and frequency grid (src/plotting.py:378-399)."""
    f = np.geomspace(freq_range_Hz[0], freq_range_Hz[1], n_pts)
    v = np.asarray(mode_shapes)[dof_idx, :]
    return f, modal_frf(frequencies_Hz, v, f, modal_damping)[0].cpu().numpy()


def modal_frf_at_dofs(frequencies_Hz, modes4, dofs, f_Hz, modal_damping=0.02):
    """FRF magnitudes (len(dofs), len(f_Hz)) straight from device-resident
    node4 modes (nmodes, NN, 4), e.g. every motor-mount DOF at once."""
    d = torch.as_tensor(np.asarray(dofs, dtype=np.int64), device=modes4.device)
    V = modes4[:, d // 3, d % 3].transpose(0, 1).to(torch.float64)      # (ndof, nmodes)
    return modal_frf(frequencies_Hz, V, f_Hz, modal_damping)
