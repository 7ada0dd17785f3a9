"""Python-3 ``Spherebin``: the scene container and binary state file of sphere.

This mirrors the hot-path subset of the reference's ``python/sphere.py``
``Spherebin`` class: the same attribute names, the same ``readbin``/``writebin``
byte layout (``python/sphere.py:254-529``, ``src/file_io.cpp:29-490``) and the
scene builders the reference's tests and examples use (``generateRadii``
:789, ``initRandomGridPos`` :1058, ``initGridAndWorldsize`` :938,
``initGridPos`` :988, ``initTemporal`` :1357, ``defaultParams`` :1391,
``bond`` :1476, ``zeroKinematics`` :1237, ``adjustUpperWall``/``adjustWall``
:1249/:1266, ``consolidate`` :1293, ``uniaxialStrainRate`` :1308, ``energy``
:1515, ``run`` :1629, ``readlast`` :783, ``status`` :2892).

Differences, all deliberate:
  * Python 3 and numpy 2 (the reference needs Python 2.7, ``numpy.infty`` and
    ``random_integers``);
  * no matplotlib/vtk imports; ``generateRadii`` draws no histogram;
  * every random draw goes through a ``numpy.random.Generator`` passed in (or
    seeded) so scenes are reproducible;
  * ``__eq__`` replaces the Python-2 ``__cmp__`` (``python/sphere.py:142-215``);
  * the fluid section (``nu > 0``) is read into ``f_v``, ``f_rho``, ``f_phi``
    and ``f_K`` (per cell, shaped as ``python/sphere.py:388-410`` makes them)
    when it holds the six values per cell that the Darcy flow writes
    (``src/file_io.cpp:466-479``); any other fluid section (the
    lattice-Boltzmann one) is kept as opaque bytes.
"""
from __future__ import annotations

import math
import os
import subprocess
from pathlib import Path

import numpy as np

_F64 = np.dtype("<f8")
_U32 = np.dtype("<u4")
_I32 = np.dtype("<i4")


def V_sphere(r):
    """Sphere volume, as ``python/sphere.py`` ``V_sphere``."""
    return 4.0 / 3.0 * math.pi * np.asarray(r) ** 3


class _Reader:
    def __init__(self, buf: bytes):
        self.buf = buf
        self.off = 0

    def take(self, dtype, count):
        dtype = np.dtype(dtype)
        n = dtype.itemsize * count
        if self.off + n > len(self.buf):
            raise ValueError(
                f"truncated sphere binary: need {n} bytes at offset {self.off}, "
                f"have {len(self.buf) - self.off}")
        out = np.frombuffer(self.buf, dtype=dtype, count=count, offset=self.off).copy()
        self.off += n
        return out


class Spherebin:
    """Scene state of one sphere simulation (``python/sphere.py:14``)."""

    def __init__(self, np_=1, nd=3, nw=1, sid="unnamed"):
        self.sid = sid
        self.nd = 3 if nd is None else int(nd)
        n = int(np_)
        self.np = n
        self.time_dt = 0.0
        self.time_current = 0.0
        self.time_total = 0.0
        self.time_file_dt = 0.0
        self.time_step_count = 0
        self.origo = np.zeros(3)
        self.L = np.zeros(3)
        self.num = np.zeros(3, dtype=np.uint32)
        self.periodic = 0
        self.x = np.zeros((n, 3))
        self.radius = np.ones(n)
        self.xysum = np.zeros((n, 2))
        self.vel = np.zeros((n, 3))
        self.fixvel = np.zeros(n)
        self.force = np.zeros((n, 3))
        self.angpos = np.zeros((n, 3))
        self.angvel = np.zeros((n, 3))
        self.torque = np.zeros((n, 3))
        self.es_dot = np.zeros(n)
        self.es = np.zeros(n)
        self.ev_dot = np.zeros(n)
        self.ev = np.zeros(n)
        self.p = np.zeros(n)
        # global parameters, defaults of python/sphere.py:70-89
        self.g = np.zeros(3)
        self.k_n = 1.16e9
        self.k_t = 1.16e9
        self.k_r = 0.0
        self.gamma_n = 0.0
        self.gamma_t = 0.0
        self.gamma_r = 0.0
        self.mu_s = 1.0
        self.mu_d = 1.0
        self.mu_r = 0.0
        self.gamma_wn = 1.0e3
        self.gamma_wt = 1.0e3
        self.mu_ws = 1.0
        self.mu_wd = 1.0
        self.rho = 2600.0
        self.contactmodel = 2
        self.kappa = 0.0
        self.db = 0.0
        self.V_b = 0.0
        # walls, python/sphere.py:96-119
        self.nw = int(nw)
        self.wmode = np.zeros(self.nw, dtype=np.int32)
        self.w_n = np.zeros((self.nw, 3))
        for i, (axis, sign) in enumerate(((2, -1.0), (0, -1.0), (0, 1.0), (1, -1.0), (1, 1.0))):
            if self.nw > i:
                self.w_n[i, axis] = sign
        self.w_x = np.ones(self.nw)
        self.w_m = np.zeros(self.nw)
        self.w_vel = np.zeros(self.nw)
        self.w_force = np.zeros(self.nw)
        self.w_devs = np.zeros(self.nw)
        self.w_devs_A = 0.0
        self.w_devs_f = 0.0
        # bonds, python/sphere.py:121-131
        self.lambda_bar = 1.0
        self.sigma_b = np.inf
        self.tau_b = np.inf
        self.bonds = np.zeros((0, 2), dtype=np.uint32)
        self.bonds_delta_n = np.zeros(0)
        self.bonds_delta_t = np.zeros((0, 3))
        self.bonds_omega_n = np.zeros(0)
        self.bonds_omega_t = np.zeros((0, 3))
        self.nu = 0.0
        self.fluid_trailer = b""
        self.f_v = self.f_rho = self.f_phi = self.f_K = None

    @property
    def nb0(self) -> int:
        return int(self.bonds.shape[0])

    # ------------------------------------------------------------------ I/O
    def to_bytes(self) -> bytes:
        """Serialise in the reference's binary layout (``src/file_io.cpp:304-490``)."""
        n, nw, nb0 = self.np, self.nw, self.nb0
        parts = [
            np.array([3], _I32), np.array([n], _U32),
            np.array([self.time_dt, self.time_current, self.time_total, self.time_file_dt], _F64),
            np.array([self.time_step_count], _U32),
            np.asarray(self.origo, _F64), np.asarray(self.L, _F64),
            np.asarray(self.num, _U32), np.array([self.periodic], _I32),
            np.column_stack([self.x, self.radius]).astype(_F64),
            np.asarray(self.xysum, _F64),
            np.column_stack([self.vel, self.fixvel]).astype(_F64),
            np.asarray(self.force, _F64), np.asarray(self.angpos, _F64),
            np.asarray(self.angvel, _F64), np.asarray(self.torque, _F64),
            np.asarray(self.es_dot, _F64), np.asarray(self.es, _F64),
            np.asarray(self.ev_dot, _F64), np.asarray(self.ev, _F64), np.asarray(self.p, _F64),
            np.asarray(self.g, _F64),
            np.array([self.k_n, self.k_t, self.k_r, self.gamma_n, self.gamma_t, self.gamma_r,
                      self.mu_s, self.mu_d, self.mu_r, self.gamma_wn, self.gamma_wt,
                      self.mu_ws, self.mu_wd, self.rho], _F64),
            np.array([self.contactmodel], _U32),
            np.array([self.kappa, self.db, self.V_b], _F64),
            np.array([nw], _U32), np.asarray(self.wmode, _I32),
            np.column_stack([self.w_n, self.w_x]).astype(_F64) if nw else np.zeros(0, _F64),
            (np.column_stack([self.w_m, self.w_vel, self.w_force, self.w_devs]).astype(_F64)
             if nw else np.zeros(0, _F64)),
            np.array([self.w_devs_A, self.w_devs_f, self.lambda_bar], _F64),
            np.array([nb0], _U32),
            np.array([self.sigma_b, self.tau_b], _F64),
            np.asarray(self.bonds, _U32),
            np.asarray(self.bonds_delta_n, _F64), np.asarray(self.bonds_delta_t, _F64),
            np.asarray(self.bonds_omega_n, _F64), np.asarray(self.bonds_omega_t, _F64),
            np.array([self.nu], _F64),
        ]
        return b"".join(np.ascontiguousarray(p).tobytes() for p in parts) + self._fluid_bytes()

    def _fluid_bytes(self) -> bytes:
        """The fluid section: per cell, z outermost and x innermost, V[3], H
        (``f_rho``), phi, K (``python/sphere.py:516-527``)."""
        if self.nu > 0.0 and self.f_v is not None:
            cells = np.concatenate([
                np.asarray(self.f_v, _F64),
                np.asarray(self.f_rho, _F64)[..., None],
                np.asarray(self.f_phi, _F64)[..., None],
                np.asarray(self.f_K, _F64)[..., None]], axis=3)        # (nx, ny, nz, 6)
            return np.ascontiguousarray(cells.transpose(2, 1, 0, 3)).tobytes()
        return self.fluid_trailer

    def writebin(self, folder="../input/", verbose=True, path=None):
        """Write ``<folder>/<sid>.bin`` (``python/sphere.py:416``)."""
        target = Path(path) if path is not None else Path(folder) / f"{self.sid}.bin"
        if verbose:
            print(f"Output file: {target}")
        target.parent.mkdir(parents=True, exist_ok=True)
        target.write_bytes(self.to_bytes())
        return target

    @classmethod
    def from_bytes(cls, buf: bytes, sid="unnamed") -> "Spherebin":
        """Parse the reference's binary layout (``src/file_io.cpp:29-301``)."""
        r = _Reader(buf)
        nd = int(r.take(_I32, 1)[0])
        if nd != 3:
            raise ValueError(f"dimensionality mismatch: dataset is {nd}D, this build is 3D")
        n = int(r.take(_U32, 1)[0])
        sb = cls(np_=n, nw=0, sid=sid)
        sb.time_dt, sb.time_current, sb.time_total, sb.time_file_dt = (float(v) for v in r.take(_F64, 4))
        sb.time_step_count = int(r.take(_U32, 1)[0])
        sb.origo = r.take(_F64, 3)
        sb.L = r.take(_F64, 3)
        sb.num = r.take(_U32, 3)
        sb.periodic = int(r.take(_I32, 1)[0])
        xr = r.take(_F64, 4 * n).reshape(n, 4)
        sb.x, sb.radius = xr[:, :3].copy(), xr[:, 3].copy()
        sb.xysum = r.take(_F64, 2 * n).reshape(n, 2)
        vf = r.take(_F64, 4 * n).reshape(n, 4)
        sb.vel, sb.fixvel = vf[:, :3].copy(), vf[:, 3].copy()
        sb.force = r.take(_F64, 3 * n).reshape(n, 3)
        sb.angpos = r.take(_F64, 3 * n).reshape(n, 3)
        sb.angvel = r.take(_F64, 3 * n).reshape(n, 3)
        sb.torque = r.take(_F64, 3 * n).reshape(n, 3)
        sb.es_dot, sb.es, sb.ev_dot, sb.ev, sb.p = (r.take(_F64, n) for _ in range(5))
        sb.g = r.take(_F64, 3)
        (sb.k_n, sb.k_t, sb.k_r, sb.gamma_n, sb.gamma_t, sb.gamma_r, sb.mu_s, sb.mu_d, sb.mu_r,
         sb.gamma_wn, sb.gamma_wt, sb.mu_ws, sb.mu_wd, sb.rho) = (float(v) for v in r.take(_F64, 14))
        sb.contactmodel = int(r.take(_U32, 1)[0])
        sb.kappa, sb.db, sb.V_b = (float(v) for v in r.take(_F64, 3))
        nw = int(r.take(_U32, 1)[0])
        if nw > 6:
            raise ValueError(f"MAXWALLS (6) is smaller than the number of walls in the file ({nw})")
        sb.nw = nw
        sb.wmode = r.take(_I32, nw)
        wn = r.take(_F64, 4 * nw).reshape(nw, 4)
        sb.w_n, sb.w_x = wn[:, :3].copy(), wn[:, 3].copy()
        wm = r.take(_F64, 4 * nw).reshape(nw, 4)
        sb.w_m, sb.w_vel, sb.w_force, sb.w_devs = (wm[:, k].copy() for k in range(4))
        sb.w_devs_A, sb.w_devs_f = (float(v) for v in r.take(_F64, 2))
        sb.lambda_bar = float(r.take(_F64, 1)[0])
        nb0 = int(r.take(_U32, 1)[0])
        sb.sigma_b, sb.tau_b = (float(v) for v in r.take(_F64, 2))
        sb.bonds = r.take(_U32, 2 * nb0).reshape(nb0, 2)
        sb.bonds_delta_n = r.take(_F64, nb0)
        sb.bonds_delta_t = r.take(_F64, 3 * nb0).reshape(nb0, 3)
        sb.bonds_omega_n = r.take(_F64, nb0)
        sb.bonds_omega_t = r.take(_F64, 3 * nb0).reshape(nb0, 3)
        sb.nu = float(r.take(_F64, 1)[0])
        sb.fluid_trailer = buf[r.off:]
        nx, ny, nz = (int(v) for v in sb.num)
        if sb.nu > 0.0 and len(sb.fluid_trailer) == 6 * 8 * nx * ny * nz:
            cells = np.frombuffer(sb.fluid_trailer, _F64).reshape(nz, ny, nx, 6)
            cells = cells.transpose(2, 1, 0, 3).copy()                 # [x, y, z, k]
            sb.f_v = cells[..., 0:3].copy()
            sb.f_rho = cells[..., 3].copy()
            sb.f_phi = cells[..., 4].copy()
            sb.f_K = cells[..., 5].copy()
            sb.fluid_trailer = b""
        return sb

    def readbin(self, targetbin, verbose=True, **_ignored):
        """Read a sphere binary into this object (``python/sphere.py:254``)."""
        if verbose:
            print(f"Input file: {targetbin}")
        other = Spherebin.from_bytes(Path(targetbin).read_bytes(), sid=self.sid)
        self.__dict__.update(other.__dict__)

    def readstep(self, step, verbose=True, root=".."):
        self.readbin(Path(root) / "output" / f"{self.sid}.output{step:05d}.bin", verbose)

    def readlast(self, verbose=True, root=".."):
        """Read the last output file of ``sid`` (``python/sphere.py:783``)."""
        self.readstep(status(self.sid, root=root), verbose, root=root)

    def __eq__(self, other):
        if not isinstance(other, Spherebin):
            return NotImplemented
        return self.to_bytes() == other.to_bytes()

    # --------------------------------------------------------- scene builders
    def generateRadii(self, psd="logn", radius_mean=440e-6, radius_variance=8.8e-9,
                      histogram=False, rng=None):
        """Random radii, log-normal or uniform (``python/sphere.py:789-823``)."""
        rng = rng or np.random.default_rng()
        if psd == "logn":
            mu = math.log((radius_mean ** 2) / math.sqrt(radius_variance + radius_mean ** 2))
            sigma = math.sqrt(math.log(radius_variance / (radius_mean ** 2) + 1))
            self.radius = rng.lognormal(mu, sigma, self.np)
        elif psd == "uni":
            self.radius = rng.uniform(radius_mean - radius_variance,
                                      radius_mean + radius_variance, self.np)
        else:
            raise ValueError(f"unknown psd {psd!r}")

    def initRandomGridPos(self, g=np.array([0.0, 0.0, -9.80665]), gridnum=np.array([12, 12, 32]),
                          periodic=1, contactmodel=2, rng=None):
        """Loose cubic configuration with random offsets (``python/sphere.py:1058-1115``)."""
        rng = rng or np.random.default_rng()
        self.g = np.asarray(g, float)
        self.periodic = int(periodic)
        coarse = np.floor(np.asarray(gridnum) / 2)
        r_max = float(np.amax(self.radius))
        cellsize = 2.1 * r_max * 2
        if (coarse[0] - 1) * (coarse[1] - 1) * (coarse[2] - 1) < self.np:
            raise NameError("Error! The grid is not sufficiently large.")
        i = np.arange(self.np)
        gp = np.stack([i % coarse[0], np.floor(i / coarse[0]) % coarse[0],
                       np.floor(i / (coarse[0] * coarse[1]))], axis=1)
        r = (self.radius * 1.05)[:, None]
        self.x = gp * cellsize + ((cellsize - r) - r) * rng.random((self.np, 3)) + r
        self.contactmodel = int(contactmodel)
        top = np.max(self.x + self.radius[:, None], axis=0)
        self.num = np.ceil(top / cellsize).astype(np.uint32)
        self.L = self.num * cellsize

    def initGridAndWorldsize(self, g=np.array([0.0, 0.0, -9.80665]), margin=2.0, periodic=1,
                             contactmodel=2):
        """World and grid around the current particles (``python/sphere.py:938-986``)."""
        self.g = np.asarray(g, float)
        self.periodic = int(periodic)
        r_max = float(np.amax(self.radius))
        self.origo = np.min(self.x - self.radius[:, None], axis=0) - margin * r_max
        self.L = np.max(self.x + self.radius[:, None], axis=0) + margin * r_max
        cellsize_min = 2.1 * r_max
        self.num = np.ceil((self.L - self.origo) / cellsize_min).astype(np.uint32)
        self.contactmodel = int(contactmodel)
        if self.nw > 0:
            self.w_x[0] = self.L[0]

    def initGridPos(self, g=np.array([0.0, 0.0, -9.80665]), gridnum=np.array([12, 12, 36]),
                    periodic=1, contactmodel=2):
        """Regular grid-like configuration (``python/sphere.py:988-1056``)."""
        self.g = np.asarray(g, float)
        self.periodic = int(periodic)
        num = np.asarray(gridnum, dtype=np.int64).copy()
        r_max = float(np.amax(self.radius))
        cellsize = 2.1 * r_max
        self.L = num * cellsize
        if num[0] * num[1] * num[2] - 8 < self.np:
            raise NameError("Error! The grid is not sufficiently large.")
        if self.periodic == 1:
            num[0] -= 1
            num[1] -= 1
        i = np.arange(self.np)
        gp = np.stack([i % num[0], np.floor(i / num[0]) % num[0],
                       np.floor(i / (num[0] * num[1]))], axis=1)
        self.x = gp * cellsize + 0.5 * cellsize
        if self.periodic == 1:
            odd = (gp[:, 2] % 2).astype(bool)
            self.x[odd, 0] += 0.5 * cellsize
            self.x[odd, 1] += 0.5 * cellsize
            num[0] += 1
            num[1] += 1
        self.num = num.astype(np.uint32)
        self.contactmodel = int(contactmodel)

    def zeroKinematics(self):
        """``python/sphere.py:1237-1247``."""
        n = self.np
        self.vel = np.zeros((n, 3))
        self.angvel = np.zeros((n, 3))
        self.angpos = np.zeros((n, 3))
        self.es = np.zeros(n)
        self.ev = np.zeros(n)
        self.xysum = np.zeros((n, 2))

    def adjustUpperWall(self, z_adjust=1.1):
        """``python/sphere.py:1249-1264``."""
        self.nw = 1
        self.wmode = np.zeros(1, dtype=np.int32)
        self.w_n = np.zeros((1, 3))
        self.w_n[0, 2] = -1.0
        self.w_vel = np.zeros(1)
        self.w_force = np.zeros(1)
        self.w_devs = np.zeros(1)
        self.w_x = np.zeros(1)
        self.w_m = np.zeros(1)
        self.adjustWall(idx=0, adjust=z_adjust)

    def adjustWall(self, idx, adjust=1.1):
        """Grid and wall placed at the particle extent (``python/sphere.py:1266-1291``)."""
        dim = {0: 2, 1: 0, 2: 0, 3: 1, 4: 1}[idx]
        xmin = float(np.min(self.x[:, dim] - self.radius))
        xmax = float(np.max(self.x[:, dim] + self.radius))
        cellsize = self.L[0] / self.num[0]
        self.num[dim] = np.uint32(np.ceil(((xmax - xmin) * adjust + xmin) / cellsize))
        self.L[dim] = (xmax - xmin) * adjust + xmin
        self.w_x[idx] = xmax if idx in (0, 1, 3) else xmin
        self.w_m[idx] = self.rho * self.np * math.pi * (cellsize / 2.0) ** 3

    def consolidate(self, deviatoric_stress=10e3, periodic=1):
        """Stress-controlled top wall (``python/sphere.py:1293-1306``)."""
        self.zeroKinematics()
        self.adjustUpperWall()
        self.wmode = np.array([1], dtype=np.int32)
        self.w_devs = np.ones(1) * deviatoric_stress

    def uniaxialStrainRate(self, wvel=-0.001, periodic=1):
        """Velocity-controlled top wall (``python/sphere.py:1308-1320``)."""
        self.zeroKinematics()
        self.adjustUpperWall()
        self.wmode = np.array([2], dtype=np.int32)
        self.w_vel = np.array([wvel])

    def initTemporal(self, total, current=0.0, file_dt=0.05, step_count=0):
        """Time step by the Zhang-Campbell rule (``python/sphere.py:1357-1377``)."""
        r_min = float(np.amin(self.radius))
        self.time_dt = 0.075 * math.sqrt((float(V_sphere(r_min)) * self.rho) / max(self.k_n, self.k_t))
        self.time_current = float(current)
        self.time_total = float(total)
        self.time_file_dt = float(file_dt)
        self.time_step_count = 0

    def defaultParams(self, mu_s=0.4, mu_d=0.4, mu_r=0.0, rho=2600, k_n=1.16e9, k_t=1.16e9,
                      k_r=0, gamma_n=0, gamma_t=0, gamma_r=0, gamma_wn=1e4, gamma_wt=1e4,
                      capillaryCohesion=0, nu=0.0):
        """``python/sphere.py:1391-1474``."""
        self.rho = float(rho)
        self.k_n, self.k_t, self.k_r = float(k_n), float(k_t), float(k_r)
        self.gamma_n, self.gamma_t, self.gamma_r = float(gamma_n), float(gamma_t), float(gamma_r)
        self.mu_s, self.mu_d, self.mu_r = float(mu_s), float(mu_d), float(mu_r)
        self.gamma_wn, self.gamma_wt = float(gamma_wn), float(gamma_wt)
        self.mu_ws, self.mu_wd = self.mu_s, self.mu_d
        theta = 0.0
        if capillaryCohesion == 1:
            self.kappa = 2.0 * math.pi * gamma_t * math.cos(theta)
            self.V_b = 1e-12
        else:
            self.kappa = 0.0
            self.V_b = 0.0
        self.db = (1.0 + theta / 2.0) * self.V_b ** (1.0 / 3.0)
        self.nu = float(nu)

    def bond(self, i, j):
        """Register a bond between particles i and j (``python/sphere.py:1476-1509``)."""
        self.lambda_bar = 1.0
        self.bonds = np.vstack([self.bonds, np.array([[i, j]], dtype=np.uint32)]).astype(np.uint32)
        self.bonds_delta_n = np.append(self.bonds_delta_n, 0.0)
        self.bonds_delta_t = np.vstack([self.bonds_delta_t, np.zeros((1, 3))])
        self.bonds_omega_n = np.append(self.bonds_omega_n, 0.0)
        self.bonds_omega_t = np.vstack([self.bonds_omega_t, np.zeros((1, 3))])

    # -------------------------------------------------------------- analysis
    def energy(self, method):
        """Sum of an energy component over all particles (``python/sphere.py:1515-1562``)."""
        m = 4.0 / 3.0 * math.pi * self.radius ** 3 * self.rho
        if method == "pot":
            return float(np.sum(m * math.sqrt(float(np.dot(self.g, self.g))) * self.x[:, 2]))
        if method == "kin":
            return float(np.sum(0.5 * m * np.sqrt(np.sum(self.vel ** 2, axis=1)) ** 2))
        if method == "rot":
            return float(np.sum(0.5 * 2.0 / 5.0 * m * self.radius ** 2
                                * np.sqrt(np.sum(self.angvel ** 2, axis=1)) ** 2))
        if method == "shear":
            return float(np.sum(self.es))
        if method == "shearrate":
            return float(np.sum(self.es_dot))
        if method == "visc_n":
            return float(np.sum(self.ev))
        if method == "visc_n_rate":
            return float(np.sum(self.ev_dot))
        if method == "bondpot":
            if self.nb0 == 0:
                return 0.0
            R_bar = self.lambda_bar * np.minimum(self.radius[self.bonds[:, 0]],
                                                 self.radius[self.bonds[:, 1]])
            A = np.pi * R_bar ** 2
            I = 0.25 * np.pi * R_bar ** 4
            J = I * 2.0
            e_fn = np.sum(0.5 * A * self.k_n * np.abs(self.bonds_delta_n) ** 2)
            e_ft = np.sum(0.5 * A * self.k_t * np.linalg.norm(self.bonds_delta_t) ** 2)
            e_tn = np.sum(0.5 * J * self.k_t * np.abs(self.bonds_omega_n) ** 2)
            e_tt = np.sum(0.5 * I * self.k_n * np.linalg.norm(self.bonds_omega_t) ** 2)
            return float(e_fn + e_ft + e_tn + e_tt)
        raise ValueError(f"unknown energy method {method!r}")

    def bulkPorosity(self):
        """``python/sphere.py:1580-1594``."""
        if self.nw == 0:
            V_total = self.L[0] * self.L[1] * self.L[2]
        else:
            V_total = self.L[0] * self.L[1] * self.w_x[0]
        V_solid = float(np.sum(V_sphere(self.radius)))
        return (V_total - V_solid) / V_total

    def run(self, verbose=True, hideinputfile=False, dry=False, root="..", binary=None):
        """Run the ``sphere`` executable on ``<root>/input/<sid>.bin``
        (``python/sphere.py:1629-1655``); the executable is this package's own
        CLI, built in-tree."""
        exe = binary or str(Path(__file__).resolve().parent / "bin" / "sphere")
        args = [exe]
        if not verbose:
            args.append("-q")
        if dry:
            args.append("--dry")
        args.append(f"input/{self.sid}.bin")
        out = subprocess.DEVNULL if hideinputfile else None
        status_ = subprocess.call(args, cwd=root, stdout=out)
        if status_ != 0:
            print(f"Warning: the sphere run returned with status {status_}")
        return status_

    def render(self, method="pres", max_val=1e3, lower_cutoff=0.0, graphicsformat="png",
               verbose=True, root="..", binary=None):
        """Render every output file of this simulation with the ray tracer
        into ``<root>/img_out/<file>.ppm`` (``python/sphere.py:1698-1725``).
        The PPM images are kept as they are: the reference's conversion to
        ``graphicsformat`` calls ImageMagick, which is not part of this build."""
        exe = binary or str(Path(__file__).resolve().parent / "bin" / "sphere")
        (Path(root) / "img_out").mkdir(exist_ok=True)
        status_ = 0
        for f in sorted((Path(root) / "output").glob(f"{self.sid}*.bin")):
            args = [exe] + ([] if verbose else ["-q"])
            if method != "normal":
                args += ["--method", method, f"{max_val}", "-l", f"{lower_cutoff}"]
            args += ["--render", str(f.relative_to(root))]
            status_ |= subprocess.call(args, cwd=root)
        return status_


def status(project, root=".."):
    """Last output-file number of a run (``python/sphere.py:2892-2907``)."""
    fn = Path(root) / "output" / f"{project}.status.dat"
    fields = fn.read_text().split()
    return int(fields[2])


def readbin(path) -> Spherebin:
    """Read a sphere binary into a new ``Spherebin``."""
    path = Path(path)
    return Spherebin.from_bytes(path.read_bytes(), sid=path.stem)
