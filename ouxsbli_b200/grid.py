"""Host-side grid, Jacobian and state conversions of the rectilinear solver.

Grids follow ``set_grid_cyclic{2,4,6}_{2D,3D}`` (src/set_coordinate.f90:120-427):
uniform spacing L / (n - 2g), node coordinates x(i) = dx*(i - g - 1) for the
interior nodes (1-based), g ghost nodes extrapolated on each side, and
cell-centred coordinates xc(i) = (x(i) + x(i+1)) / 2.
"""
from __future__ import annotations

import numpy as np


def cyclic_axis(n: int, L: float, order: int) -> tuple[np.ndarray, np.ndarray]:
    """Cell-centre coordinates (n) and spacings (n-1) of one periodic axis."""
    g = order // 2
    d1 = L / float(n - 2 * g)
    x = np.zeros(n + 1)
    lo, hi = g + 1, n - g + 1  # 1-based interior node range
    for i in range(lo, hi + 1):
        x[i - 1] = d1 * float(i - lo)
    for m in range(1, g + 1):
        x[lo - 1 - m] = x[lo - 1] - float(m) * d1
        x[hi - 1 + m] = x[hi - 1] + float(m) * d1
    xc = 0.5 * (x[:-1] + x[1:])
    return xc, np.full(n - 1, d1)


def jacobian(dx: np.ndarray, dy: np.ndarray, dz: np.ndarray | None) -> np.ndarray:
    """J(nx, ny) = 1 / cell volume with copied edges (set_Jacobian_xy{2,3}).

    Returned in Fortran order (J[i, j] with i fastest in memory)."""
    nx, ny = dx.size + 1, dy.size + 1
    J = np.zeros((nx, ny), order="F")
    for j in range(1, ny - 1):
        for i in range(1, nx - 1):
            if dz is not None:
                J[i, j] = 8.0 / ((dx[i - 1] + dx[i]) * (dy[j - 1] + dy[j]) * 2.0 * dz[0])
            else:
                J[i, j] = 4.0 / ((dx[i - 1] + dx[i]) * (dy[j - 1] + dy[j]))
    J[:, 0] = J[:, 1]
    J[:, ny - 1] = J[:, ny - 2]
    J[0, :] = J[1, :]
    J[nx - 1, :] = J[nx - 2, :]
    return J


def fill_periodic(Q: np.ndarray, g: int) -> None:
    """Periodic ghost images for Q[nx, nv, ny(, nz)] in place (set_bc_cyclic*_init)."""
    dim = Q.ndim - 1
    if dim == 3:
        nx, _, ny, nz = Q.shape
    else:
        nx, _, ny = Q.shape
        nz = 1
    ix = (np.arange(nx) - g) % (nx - 2 * g) + g
    iy = (np.arange(ny) - g) % (ny - 2 * g) + g
    if dim == 3:
        iz = (np.arange(nz) - g) % (nz - 2 * g) + g
        Q[...] = Q[ix][:, :, iy][:, :, :, iz]
    else:
        Q[...] = Q[ix][:, :, iy]


def to_qj(Q: np.ndarray, J: np.ndarray) -> np.ndarray:
    """Q / J in the reference's layout (pre_calc, preprocess.f90.fypp:64-72)."""
    if Q.ndim == 4:
        return np.asfortranarray(Q / J[:, None, :, None])
    return np.asfortranarray(Q / J[:, None, :])


def from_qj(QJ: np.ndarray, J: np.ndarray) -> np.ndarray:
    """J * QJ, the conservative variables written to recal/Q00001.dat (main.f90:82-93)."""
    if QJ.ndim == 4:
        return np.asfortranarray(J[:, None, :, None] * QJ)
    return np.asfortranarray(J[:, None, :] * QJ)
