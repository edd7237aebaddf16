"""NumPy model of the library's multigrid hierarchy (test helper).

Same coarsening rule (each axis with >= 2 elements halves, ceil; axes of one
element are kept; stop at <= 160 nodes) and the same trilinear prolongation,
so the device's Galerkin coarse operators can be checked against an explicit
P^T (D K D) P built from the oracle's assembled stiffness.
"""
import numpy as np
import scipy.sparse as sp


def levels(nx, ny, nz, cap=160):
    L = [(nx, ny, nz, 1, 1, 1)]
    while True:
        nx, ny, nz = L[-1][:3]
        if (nx + 1) * (ny + 1) * (nz + 1) <= cap or (nx < 2 and ny < 2 and nz < 2):
            return L
        f = [2 if n >= 2 else 1 for n in (nx, ny, nz)]
        L.append(((nx + f[0] - 1) // f[0], (ny + f[1] - 1) // f[1], (nz + f[2] - 1) // f[2], *f))


def _axis(nf, nc, f):
    rows, cols, vals = [], [], []
    for i in range(nf):
        if f == 1:
            rows.append(i); cols.append(i); vals.append(1.0)
        elif i % 2 == 0:
            rows.append(i); cols.append(i // 2); vals.append(1.0)
        else:
            rows += [i, i]; cols += [(i - 1) // 2, (i + 1) // 2]; vals += [0.5, 0.5]
    return sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))


def prolongation(fine, coarse):
    """DOF prolongation (3 NN_f x 3 NN_c), node index k*NX*NY + j*NX + i."""
    nx, ny, nz = fine[:3]
    cx, cy, cz, fx, fy, fz = coarse
    Pn = sp.kron(_axis(nz + 1, cz + 1, fz), sp.kron(_axis(ny + 1, cy + 1, fy), _axis(nx + 1, cx + 1, fx)))
    return sp.kron(Pn, sp.eye(3)).tocsr()


def assemble_elements(Ae, nx, ny, nz):
    """Global matrix from per-element 24x24 matrices (reference local order)."""
    NX, NY = nx + 1, ny + 1
    di = np.array([0, 1, 1, 0, 0, 1, 1, 0])
    dj = np.array([0, 0, 1, 1, 0, 0, 1, 1])
    dk = np.array([0, 0, 0, 0, 1, 1, 1, 1])
    EZ, EY, EX = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    EX, EY, EZ = EX.ravel(), EY.ravel(), EZ.ravel()
    nodes = (EZ[:, None] + dk) * NX * NY + (EY[:, None] + dj) * NX + (EX[:, None] + di)
    dofs = (3 * nodes[:, :, None] + np.arange(3)).reshape(-1, 24)
    rr = np.repeat(dofs, 24, axis=1).ravel()
    cc = np.tile(dofs, (1, 24)).ravel()
    n = 3 * NX * NY * (nz + 1)
    return sp.coo_matrix((np.asarray(Ae, float).reshape(-1), (rr, cc)), shape=(n, n)).tocsr()
