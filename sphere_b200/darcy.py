"""Host side of the Darcy flow (the reference's ``DEM::d`` arrays,
src/darcy.cpp:17-38, src/datatypes.h).

The fluid grid is the cell grid with one ghost node on every side:
(nx+2)(ny+2)(nz+2) nodes, x fastest, node (x, y, z) at
(x+1) + (nx+2)(y+1) + (nx+2)(ny+2)(z+1) for -1 <= x <= nx and so on.  Every
field holds one double per node, V, dH and T three.  These are the arrays
``Simulation.darcy_upload`` / ``darcy_download`` exchange with the device and
that the input file's fluid section fills (V, H, phi, K of every cell).
"""
from __future__ import annotations

from dataclasses import dataclass, fields

import numpy as np


@dataclass
class DarcyState:
    H: np.ndarray        # hydraulic pressure
    H_new: np.ndarray    # the pressure's second buffer
    V: np.ndarray        # (n, 3) pore velocity
    dH: np.ndarray       # (n, 3) pressure gradient
    K: np.ndarray        # hydraulic conductivity
    T: np.ndarray        # (n, 3) transmissivity
    Ss: np.ndarray       # specific storativity
    W: np.ndarray        # recharge
    phi: np.ndarray      # porosity
    dphi: np.ndarray     # porosity change in the last step
    num: tuple = (0, 0, 0)

    @staticmethod
    def zeros(num) -> "DarcyState":
        """Every node zero: the reference leaves the arrays it does not read
        from the file unset; this build reads them as zero."""
        nx, ny, nz = (int(v) for v in num)
        n = (nx + 2) * (ny + 2) * (nz + 2)
        one = lambda: np.zeros(n)          # noqa: E731
        three = lambda: np.zeros((n, 3))   # noqa: E731
        return DarcyState(H=one(), H_new=one(), V=three(), dH=three(), K=one(), T=three(),
                          Ss=one(), W=one(), phi=one(), dphi=one(), num=(nx, ny, nz))

    def copy(self) -> "DarcyState":
        return DarcyState(**{f.name: (getattr(self, f.name).copy()
                                      if isinstance(getattr(self, f.name), np.ndarray)
                                      else getattr(self, f.name)) for f in fields(self)})

    def node(self, x, y, z):
        """Flat index of node (x, y, z); ghosts at -1 and num."""
        nx, ny, _ = self.num
        return (np.asarray(x) + 1) + (nx + 2) * (np.asarray(y) + 1) + \
            (nx + 2) * (ny + 2) * (np.asarray(z) + 1)

    def interior(self, name: str) -> np.ndarray:
        """Field `name` over the cells only, indexed [z, y, x] (a copy)."""
        nx, ny, nz = self.num
        a = getattr(self, name)
        shape = (nz + 2, ny + 2, nx + 2) + a.shape[1:]
        return a.reshape(shape)[1:-1, 1:-1, 1:-1].copy()

    def set_cells(self, V=None, H=None, phi=None, K=None):
        """Fill the cells (not the ghosts) from per-cell arrays shaped
        (nx, ny, nz[, 3]), the layout of the input file's fluid section."""
        nx, ny, nz = self.num
        xs, ys, zs = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        idx = self.node(xs, ys, zs)
        for name, val in (("V", V), ("H", H), ("phi", phi), ("K", K)):
            if val is not None:
                getattr(self, name)[idx] = val

    def cells(self, name: str) -> np.ndarray:
        """Field `name` over the cells, shaped (nx, ny, nz[, 3])."""
        nx, ny, nz = self.num
        xs, ys, zs = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
        return getattr(self, name)[self.node(xs, ys, zs)]

    @staticmethod
    def from_spherebin(sb) -> "DarcyState":
        """The grid as the reference's readbin leaves it (src/file_io.cpp:
        270-292): V, H, phi and K of every cell from the file's fluid
        section, everything else zero."""
        ds = DarcyState.zeros(sb.num)
        if sb.f_v is not None:
            ds.set_cells(V=sb.f_v, H=sb.f_rho, phi=sb.f_phi, K=sb.f_K)
        return ds

    def to_spherebin(self, sb):
        """Write V, H, phi, K of every cell into the file's fluid section."""
        sb.f_v, sb.f_rho = self.cells("V"), self.cells("H")
        sb.f_phi, sb.f_K = self.cells("phi"), self.cells("K")
        sb.fluid_trailer = b""

    def arrays(self):
        return {f.name: getattr(self, f.name) for f in fields(self) if f.name != "num"}
