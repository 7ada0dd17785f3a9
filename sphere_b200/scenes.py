"""Seeded synthetic scenes for the DEM hot path.

Each builder returns a ``Spherebin`` (reference binary layout) built from a
``numpy.random.default_rng(seed)``; no dataset is involved.  The workloads:

``settling``      10,000 monodisperse spheres (r = 0.01 m, rho = 2600) on a
                  jittered cubic lattice (spacing 2.2 r, 20 x 20 x 25,
                  jitter U(+-0.1 r)) in a 0.5 x 0.5 x 2 m box with the
                  reference's implicit frictional walls, gravity -9.81 m/s^2,
                  linear-viscoelastic contacts (kn = kt = 1e6 N/m,
                  gamma_n = 100 N s/m, mu = 0.5), dt = 1e-6 s, grid 24 x 24 x 96.
``polydisperse``  1,000,000 spheres, radii log-normal (median 1 mm,
                  sigma 0.2, clipped to 0.5-2 mm), random sequential placement
                  in a periodic-x/y 0.2 x 0.2 x 0.4 m domain, a top wall at
                  max(z + r) loaded at 20 kPa, contact parameters of
                  ``settling`` plus mu_r = 0.01 (unused by contact model 2),
                  dt = 2e-7 s, grid 50 x 50 x 100.
``bonded``        uniform radii 0.9-1.1 mm on a jittered FCC lattice with a
                  bond between every lattice-neighbour pair, both x ends
                  pulled apart at 0.01 m/s (``fixvel``).
``collision``     small dense scenes with random velocities and spins, used
                  by the parity tests because every step makes and breaks
                  contacts and slides.
"""
from __future__ import annotations

import math

import numpy as np

from .spherebin import Spherebin, V_sphere


def _contact_params(sb: Spherebin, k_n=1e6, k_t=1e6, gamma_n=100.0, gamma_t=0.0, mu=0.5,
                    gamma_w=100.0, mu_r=0.0):
    sb.k_n, sb.k_t, sb.k_r = float(k_n), float(k_t), 0.0
    sb.gamma_n, sb.gamma_t, sb.gamma_r = float(gamma_n), float(gamma_t), 0.0
    sb.mu_s = sb.mu_d = sb.mu_ws = sb.mu_wd = float(mu)
    sb.mu_r = float(mu_r)
    sb.gamma_wn = sb.gamma_wt = float(gamma_w)
    sb.rho = 2600.0
    sb.contactmodel = 2
    sb.kappa = sb.db = sb.V_b = 0.0


def settling(seed=0, nx=20, ny=20, nz=25, r=0.01, sid="settling") -> Spherebin:
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    sb = Spherebin(np_=n, nw=0, sid=sid)
    spacing = 2.2 * r
    i = np.arange(n)
    lat = np.stack([i % nx, (i // nx) % ny, i // (nx * ny)], axis=1).astype(float)
    sb.x = 0.03 + lat * spacing + rng.uniform(-0.1 * r, 0.1 * r, size=(n, 3))
    sb.radius = np.full(n, r)
    sb.origo = np.zeros(3)
    sb.L = np.array([0.5, 0.5, 2.0])
    sb.num = np.array([24, 24, 96], dtype=np.uint32)
    sb.periodic = 0
    sb.g = np.array([0.0, 0.0, -9.81])
    _contact_params(sb)
    sb.time_dt = 1e-6
    sb.time_total = 1000 * sb.time_dt
    sb.time_file_dt = sb.time_total
    return sb


def _lognormal_radii(rng, n, median=1e-3, sigma=0.2, lo=0.5e-3, hi=2e-3):
    return np.clip(np.exp(rng.normal(math.log(median), sigma, n)), lo, hi)


def _scenegen():
    import ctypes as C
    from pathlib import Path
    from . import build
    path = build.build_scenegen()
    lib = C.CDLL(str(path))
    lib.rsa_place.argtypes = [C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                              C.POINTER(C.c_double), C.c_int, C.c_uint64, C.c_int64,
                              C.POINTER(C.c_double)]
    lib.rsa_place.restype = C.c_int
    return lib


def rsa_place(rng, radii, L, periodic_xy=True, max_trials=10_000_000):
    """Random sequential placement of spheres with the given radii in the box
    [0, L): largest spheres first (ties in index order), each at uniformly
    random positions until it overlaps no placed sphere (periodic images in
    x/y, hard floor/ceiling in z).  The placement runs in native code
    (csrc/host/scenegen.c) from a seed drawn from ``rng``.  Returns (n, 3)."""
    import ctypes as C
    radii = np.ascontiguousarray(radii, dtype=np.float64)
    Larr = np.ascontiguousarray(L, dtype=np.float64)
    pos = np.zeros((len(radii), 3))
    seed = int(rng.integers(0, 2**63 - 1))
    order = np.ascontiguousarray(np.argsort(-radii, kind="stable"), dtype=np.int64)
    dp = C.POINTER(C.c_double)
    rc = _scenegen().rsa_place(len(radii), radii.ctypes.data_as(dp),
                               order.ctypes.data_as(C.POINTER(C.c_int64)), Larr.ctypes.data_as(dp),
                               1 if periodic_xy else 0, seed, int(max_trials),
                               pos.ctypes.data_as(dp))
    if rc != 0:
        raise RuntimeError(f"rsa_place failed ({rc}): the packing is too dense for RSA")
    return pos


def polydisperse(n=1_000_000, seed=0, L=(0.2, 0.2, 0.4), num=(50, 50, 100),
                 devs=20e3, sid="polydisperse") -> Spherebin:
    rng = np.random.default_rng(seed)
    sb = Spherebin(np_=n, nw=1, sid=sid)
    sb.radius = _lognormal_radii(rng, n)
    sb.x = rsa_place(rng, sb.radius, L)
    sb.origo = np.zeros(3)
    sb.L = np.array(L, float)
    sb.num = np.array(num, dtype=np.uint32)
    sb.periodic = 1
    sb.g = np.array([0.0, 0.0, -9.81])
    _contact_params(sb, mu_r=0.01)
    # stress-controlled top wall at max(z + r) (python/sphere.py:1266-1306)
    sb.nw = 1
    sb.wmode = np.array([1], dtype=np.int32)
    sb.w_n = np.array([[0.0, 0.0, -1.0]])
    sb.w_x = np.array([float(np.max(sb.x[:, 2] + sb.radius))])
    cellsize = sb.L[0] / sb.num[0]
    sb.w_m = np.array([sb.rho * n * math.pi * (cellsize / 2.0) ** 3])
    sb.w_vel = np.zeros(1)
    sb.w_force = np.zeros(1)
    sb.w_devs = np.array([devs])
    sb.time_dt = 2e-7
    sb.time_total = 1e4 * sb.time_dt
    sb.time_file_dt = sb.time_total
    return sb


def packed(nx=100, ny=100, nz=100, r=1e-3, sigma=20e3, seed=0, height=0.4,
           sid="packed") -> Spherebin:
    """A jammed simple-cubic column: every sphere presses on its six lattice
    neighbours, so each holds six contacts through the whole run
    (C ~ 6 N directed contacts, the packed-bed coordination number).

    - nx x ny x nz spheres of radius r (1 mm), density 2600 kg/m^3;
    - lattice spacing 2 r - delta, delta = sigma s^2 / k_n, the overlap at
      which the contact force carries the wall's normal stress sigma over
      one lattice site (8e-8 m at 20 kPa and k_n = 1e6 N/m);
    - x and y periodic with the period equal to the lattice, so contacts
      cross the periodic faces too; the floor at z = 0 and a stress-
      controlled top wall (20 kPa) each overlap their layer by delta;
    - contact parameters of ``polydisperse`` and its dt (2e-7 s), except the
      viscosities.  gamma_n is 0: contact model 2's normal viscosity
      (src/contactmodels.cuh, f_n = (-k_n delta - gamma_n vel_n) n with
      vel_n = -dv.n) lowers the push between approaching spheres and raises
      it between separating ones, so in a lattice that vibrates it feeds
      energy in at a rate of about gamma_n / m, and any gamma_n above zero
      blows the column up within a few hundred steps.  The wall viscosities
      are 0.48 of critical for one contact (the damping ratio of
      ``settling``): at 100 N s/m, the value of the other scenes, the wall's
      tangential damping of a 1 mm sphere's spin (gamma r^2 dt / I = 4.6) is
      past the explicit step's stability limit;
    - a seeded jitter of delta / 100 breaks the lattice's exact symmetry.

    The grid is two lattice sites per cell in x and y and 4 mm cells in z."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    k_n = 1e6
    m = 2600.0 * float(V_sphere(r))
    gamma_w = 0.48 * 2.0 * math.sqrt(k_n * m)
    s0 = 2.0 * r
    delta = sigma * s0 * s0 / k_n
    s = s0 - delta
    sb = Spherebin(np_=n, nw=1, sid=sid)
    i = np.arange(n)
    lat = np.stack([i % nx, (i // nx) % ny, i // (nx * ny)], axis=1).astype(float)
    sb.x = lat * s + np.array([0.5 * s, 0.5 * s, r - delta])
    sb.x += rng.uniform(-0.01 * delta, 0.01 * delta, size=(n, 3))
    sb.radius = np.full(n, r)
    sb.origo = np.zeros(3)
    sb.L = np.array([nx * s, ny * s, float(height)])
    sb.num = np.array([nx // 2, ny // 2, int(height / (4.0 * r))], dtype=np.uint32)
    sb.periodic = 1
    sb.g = np.array([0.0, 0.0, -9.81])
    _contact_params(sb, gamma_n=0.0, gamma_w=gamma_w, mu_r=0.01)
    sb.nw = 1
    sb.wmode = np.array([1], dtype=np.int32)
    sb.w_n = np.array([[0.0, 0.0, -1.0]])
    sb.w_x = np.array([float(np.max(sb.x[:, 2])) + r - delta])
    sb.w_m = np.array([m * nx * ny])
    sb.w_vel = np.zeros(1)
    sb.w_force = np.zeros(1)
    sb.w_devs = np.array([float(sigma)])
    sb.time_dt = 2e-7
    sb.time_total = 1e4 * sb.time_dt
    sb.time_file_dt = sb.time_total
    return sb


def bonded(seed=0, nx=40, ny=20, nz=20, r_lo=0.9e-3, r_hi=1.1e-3, pull=0.01,
           sigma_b=2e7, tau_b=2e7, spacing=None, bond_all=False, sid="bonded") -> Spherebin:
    """FCC lattice with the nearest-neighbour distance `spacing` (default the
    mean diameter: a close packing, where pairs with ri + rj above it
    overlap), bonds between all pairs closer than 1.05 (ri + rj), or with
    `bond_all` between every pair of lattice neighbours; the first and last x
    layer move apart at +-pull/2."""
    rng = np.random.default_rng(seed)
    nn_dist = (r_lo + r_hi) if spacing is None else float(spacing)
    a = nn_dist * math.sqrt(2.0)   # cubic FCC cell edge
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"),
                     axis=-1).reshape(-1, 3)
    pts = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    order = np.lexsort((pts[:, 0], pts[:, 1], pts[:, 2]))
    pts = pts[order]
    n = len(pts)
    sb = Spherebin(np_=n, nw=0, sid=sid)
    sb.radius = rng.uniform(r_lo, r_hi, n)
    margin = 4 * r_hi
    sb.x = pts + margin + rng.uniform(-0.02 * r_lo, 0.02 * r_lo, size=(n, 3))
    ext = pts.max(axis=0) + 2 * margin
    cell = 2.2 * r_hi
    num = np.ceil(ext / cell).astype(np.uint32)
    sb.origo = np.zeros(3)
    sb.L = num * cell
    sb.num = num
    sb.periodic = 0
    sb.g = np.zeros(3)
    _contact_params(sb, k_n=1e6, k_t=1e6, gamma_n=0.0, mu=0.5)
    # bonds: lattice neighbours at the FCC nearest-neighbour distance
    nn = a / math.sqrt(2.0)
    key = np.floor(sb.x / cell).astype(np.int64)
    kid = key[:, 0] + num[0] * (key[:, 1] + num[1] * key[:, 2])
    srt = np.argsort(kid, kind="stable")
    skid = kid[srt]
    pairs = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                nk = (key[:, 0] + dx) + num[0] * ((key[:, 1] + dy) + num[1] * (key[:, 2] + dz))
                lo = np.searchsorted(skid, nk, "left")
                hi = np.searchsorted(skid, nk, "right")
                cnt = hi - lo
                src = np.repeat(np.arange(n), cnt)
                oth = srt[np.repeat(lo, cnt) + (np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt))]
                sel = oth > src
                src, oth = src[sel], oth[sel]
                d = np.linalg.norm(sb.x[src] - sb.x[oth], axis=1)
                ok = d < 1.2 * nn
                if not bond_all:
                    ok &= d < 1.05 * (sb.radius[src] + sb.radius[oth])
                pairs.append(np.stack([src[ok], oth[ok]], axis=1))
    bonds = np.unique(np.concatenate(pairs), axis=0).astype(np.uint32)
    sb.bonds = bonds
    nb0 = len(bonds)
    sb.lambda_bar = 1.0
    sb.bonds_delta_n = np.zeros(nb0)
    sb.bonds_delta_t = np.zeros((nb0, 3))
    sb.bonds_omega_n = np.zeros(nb0)
    sb.bonds_omega_t = np.zeros((nb0, 3))
    sb.sigma_b, sb.tau_b = float(sigma_b), float(tau_b)
    xmin, xmax = sb.x[:, 0].min(), sb.x[:, 0].max()
    left = sb.x[:, 0] < xmin + 0.5 * a
    right = sb.x[:, 0] > xmax - 0.5 * a
    sb.fixvel[left | right] = 1.0
    sb.vel[left, 0] = -0.5 * pull
    sb.vel[right, 0] = 0.5 * pull
    m_min = float(V_sphere(r_lo)) * sb.rho
    sb.time_dt = 1e-7
    sb.time_total = 1000 * sb.time_dt
    sb.time_file_dt = sb.time_total
    _ = m_min
    return sb


def tension(nx=62, ny=32, nz=32, seed=0, pull=0.01, sigma_b=0.003, tau_b=0.003,
            sid="tension") -> Spherebin:
    """The bonded-tension workload: a bar of nx x ny x nz FCC cells (4
    spheres each; 253,952 at the default 62 x 32 x 32, 0.20 x 0.10 x 0.10 m)
    laid along x, radii U(0.9, 1.1) mm, a bond between every pair of lattice
    neighbours (12 per sphere, about 6 per sphere counted once), both x end
    layers pulled apart at pull/2 each, dt = 1e-7 s, no gravity.

    The lattice spacing is 2.25 mm, the largest diameter plus the jitter
    of the positions on both sides, so no pair overlaps
    at the start: the reference's bonds are as stiff as k_n A (a few N/m at
    k_n = 1e6 N/m and the bond section A = pi (0.9 mm)^2), against the
    contacts' 1e6 N/m, so a packing whose neighbours overlap flies apart
    under its contact forces before any pull acts.  Bond stiffness is the
    reference's k_n A and k_t A (contact k_n = k_t = 1e6 N/m).

    The bar starts in homogeneous stretch: x velocities linear in x, from
    -pull/2 at one end layer to +pull/2 at the other.  Pulled at its ends
    from rest, the bar (whose longitudinal wave speed with these bonds is
    about 1 m/s) would tear at the end layers and nowhere else within the
    run; stretched as a whole, every bond lengthens at 0.05 / s times its
    length, and the breaking strengths sigma_b = tau_b = 0.003 (the
    reference's units: k_n times the stretch, plus bending) are reached
    throughout the bar after about 600 steps, where about 70% of the bonds
    (those along the pull) break."""
    sb = bonded(seed=seed, nx=nx, ny=ny, nz=nz, pull=pull, sigma_b=sigma_b, tau_b=tau_b,
                spacing=2.25e-3, bond_all=True, sid=sid)
    x = sb.x[:, 0]
    lo, hi = float(x.min()), float(x.max())
    sb.vel[:, 0] = pull * ((x - lo) / (hi - lo) - 0.5)
    ends = sb.fixvel > 0
    sb.vel[ends, 0] = np.where(x[ends] < 0.5 * (lo + hi), -0.5 * pull, 0.5 * pull)
    return sb


def collision(n=2000, seed=0, periodic=0, box=(0.06, 0.06, 0.06), r=(0.8e-3, 1.6e-3),
              phi_target=0.45, nw=0, vmax=0.5, wmax=200.0, g=(0.0, 0.0, -9.81),
              k_n=2e4, k_t=2e4, gamma_n=0.05, gamma_t=0.01, mu=0.4, dt=2e-6,
              straddle=False, sid="collision") -> Spherebin:
    """Jittered lattice with some overlap, random velocities and spins:
    contacts open, close and slide from the first step on.  The box is sized
    so no particle reaches a periodic boundary within a few hundred steps,
    unless ``straddle`` moves the cluster across the x and y boundaries (with
    periodic x/y, particles then leave and re-enter the grid every few steps)."""
    rng = np.random.default_rng(seed)
    radii = rng.uniform(r[0], r[1], n)
    vol = float(np.sum(V_sphere(radii)))
    side = (vol / phi_target) ** (1.0 / 3.0)
    m = int(math.ceil(n ** (1.0 / 3.0)))
    spacing = side / m
    i = np.arange(n)
    lat = np.stack([i % m, (i // m) % m, i // (m * m)], axis=1).astype(float)
    Lb = np.asarray(box, float)
    center = 0.5 * Lb
    x = center - 0.5 * side + (lat + 0.5) * spacing + rng.uniform(-0.15, 0.15, (n, 3)) * spacing
    if straddle:
        x[:, :2] = np.mod(x[:, :2] + 0.5 * Lb[:2], Lb[:2])
    sb = Spherebin(np_=n, nw=nw, sid=sid)
    sb.radius = radii
    sb.x = x
    sb.vel = rng.uniform(-vmax, vmax, (n, 3))
    sb.angvel = rng.uniform(-wmax, wmax, (n, 3))
    sb.origo = np.zeros(3)
    sb.L = Lb
    cell = 2.0 * r[1]
    sb.num = np.floor(Lb / cell).astype(np.uint32)
    sb.periodic = int(periodic)
    sb.g = np.asarray(g, float)
    _contact_params(sb, k_n=k_n, k_t=k_t, gamma_n=gamma_n, gamma_t=gamma_t, mu=mu, gamma_w=0.05)
    if nw:
        sb.wmode = np.ones(nw, dtype=np.int32)
        sb.w_x = np.array([float(np.max(sb.x[:, 2] + sb.radius)) - 0.05e-3] + [0.0] * (nw - 1))[:nw]
        sb.w_m = np.full(nw, 1e-3)
        sb.w_devs = np.full(nw, 50.0)
    sb.time_dt = dt
    sb.time_total = 100 * dt
    sb.time_file_dt = sb.time_total
    return sb


def ensemble_member(i, cell_factor=2.0, n_range=(500, 20000), sid=None) -> Spherebin:
    """Member i of the batched settling ensemble, seeded by 1000 + i.

    - particle count N = round(exp(U(ln 500, ln 20000)));
    - radii U(0.9, 1.1) mm, density 2600 kg/m^3;
    - mu_s = mu_d = mu_ws = mu_wd ~ U(0.2, 0.8);
    - k_n = k_t log-uniform in [1e5, 1e7] N/m.

    The layout is ``settling`` scaled to N: a jittered cubic lattice (spacing
    2.2 r_max, jitter U(+-0.1 r), nz ~ 1.25 nx) with 3 r_max margins in a box
    3.6 times as tall as the lattice, implicit frictional walls, gravity
    -9.81 m/s^2.  The time step follows the reference's rule
    0.075 sqrt(m_min / max(k_n, k_t)) (python/sphere.py:1371).  gamma_n is
    0.48 of the critical 2 sqrt(m k_n) at the 1 mm mass, the damping ratio of
    ``settling``, and the wall damping equals it.  Cells are at least
    ``cell_factor`` r_max wide."""
    rng = np.random.default_rng(1000 + i)
    n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
    radii = rng.uniform(0.9e-3, 1.1e-3, n)
    mu = float(rng.uniform(0.2, 0.8))
    k = float(math.exp(rng.uniform(math.log(1e5), math.log(1e7))))
    r_max = float(radii.max())
    spacing = 2.2 * r_max
    nx = max(3, int(round((n / 1.25) ** (1.0 / 3.0))))
    nz = int(math.ceil(n / (nx * nx)))
    idx = np.arange(n)
    lat = np.stack([idx % nx, (idx // nx) % nx, idx // (nx * nx)], axis=1).astype(float)
    margin = 3.0 * r_max
    sb = Spherebin(np_=n, nw=0, sid=sid or f"ensemble{i:04d}")
    sb.radius = radii
    sb.x = margin + lat * spacing + rng.uniform(-0.1, 0.1, (n, 3)) * radii[:, None]
    width = 2.0 * margin + (nx - 1) * spacing
    height = 3.6 * (2.0 * margin + (nz - 1) * spacing)
    sb.origo = np.zeros(3)
    sb.L = np.array([width, width, height])
    sb.num = np.maximum(3, np.floor(sb.L / (cell_factor * r_max))).astype(np.uint32)
    sb.periodic = 0
    sb.g = np.array([0.0, 0.0, -9.81])
    m_ref = 4.0 / 3.0 * math.pi * 1e-3 ** 3 * 2600.0
    gamma_n = 0.48 * 2.0 * math.sqrt(m_ref * k)
    _contact_params(sb, k_n=k, k_t=k, gamma_n=gamma_n, gamma_t=0.0, mu=mu, gamma_w=gamma_n)
    m_min = 4.0 / 3.0 * math.pi * float(radii.min()) ** 3 * sb.rho
    sb.time_dt = 0.075 * math.sqrt(m_min / k)
    sb.time_total = 2000 * sb.time_dt
    sb.time_file_dt = sb.time_total
    return sb


def jammed_member(i, n_range=(500, 20000), r=1e-3, sigma=20e3, sid=None) -> Spherebin:
    """Member i of the contact-laden ensemble: ``packed`` at the member's
    size, so that every sphere holds about six contacts from the first step.

    - the particle count and the stiffness and friction draws of
      ``ensemble_member`` i (seed 1000 + i): N log-uniform in 500-20,000,
      k_n = k_t log-uniform in 1e5-1e7 N/m, mu ~ U(0.2, 0.8);
    - a simple-cubic lattice nx x nx x nz (nx ~ (N / 1.25)^(1/3)) of spheres
      of radius r = 1 mm (one radius: a lattice of unequal spheres cannot be
      jammed evenly), spacing 2 r - delta with delta = sigma (2 r)^2 / k_n,
      the overlap that carries a 20 kPa stress;
    - periodic x/y with the lattice's period; the floor and the top of the
      box (the reference's implicit walls, no dynamic wall: batched scenes
      have none) each overlap their layer by delta;
    - no normal viscosity (contact model 2's normal viscosity drives a
      vibrating lattice apart, see ``packed``), wall viscosities 0.48 of
      critical, dt = 0.075 sqrt(m / k_n) (python/sphere.py:1371), gravity
      -9.81 m/s^2."""
    rng = np.random.default_rng(1000 + i)
    n_draw = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
    rng.uniform(0.9e-3, 1.1e-3, n_draw)   # the radii draw of ensemble_member, unused
    mu = float(rng.uniform(0.2, 0.8))
    k = float(math.exp(rng.uniform(math.log(1e5), math.log(1e7))))
    nx = max(6, int(round((n_draw / 1.25) ** (1.0 / 3.0))))
    nz = max(2, int(round(n_draw / (nx * nx))))
    n = nx * nx * nz
    m = 2600.0 * float(V_sphere(r))
    s0 = 2.0 * r
    delta = sigma * s0 * s0 / k
    spacing = s0 - delta
    sb = Spherebin(np_=n, nw=0, sid=sid or f"jammed{i:04d}")
    idx = np.arange(n)
    lat = np.stack([idx % nx, (idx // nx) % nx, idx // (nx * nx)], axis=1).astype(float)
    sb.x = lat * spacing + np.array([0.5 * spacing, 0.5 * spacing, r - delta])
    sb.x += rng.uniform(-0.01 * delta, 0.01 * delta, size=(n, 3))
    sb.radius = np.full(n, r)
    sb.origo = np.zeros(3)
    top = r - delta + (nz - 1) * spacing
    sb.L = np.array([nx * spacing, nx * spacing, top + r - delta])
    sb.num = np.array([nx // 2, nx // 2, max(1, int(sb.L[2] / (2.2 * r)))], dtype=np.uint32)
    sb.periodic = 1
    sb.g = np.array([0.0, 0.0, -9.81])
    gamma_w = 0.48 * 2.0 * math.sqrt(k * m)
    _contact_params(sb, k_n=k, k_t=k, gamma_n=0.0, gamma_t=0.0, mu=mu, gamma_w=gamma_w)
    sb.time_dt = 0.075 * math.sqrt(m / k)
    sb.time_total = 2000 * sb.time_dt
    sb.time_file_dt = sb.time_total
    return sb


def jammed_column(nx=40, ny=40, nz=63, r=1e-3, sigma=20e3, k=1e6, mu=0.3, vmax=0.005,
                  wmax=20.0, gamma_frac=1e-3, dt=5e-7, seed=0, sid="jammed_column") -> Spherebin:
    """The calibration column in contact from the first step: a jammed
    simple-cubic block of nx x ny x nz spheres (100,800 at the default, 8 x 8
    x 12.6 cm), r = 1 mm, spacing 2 r - delta (delta = sigma (2 r)^2 / k, the
    overlap that carries a 20 kPa stress), held in a box of its own size by
    the reference's six implicit frictional walls, each overlapping its layer
    by delta (a free block would spring apart: its contacts only push).  It
    is stirred: seeded velocities U(+-vmax) and spins U(+-wmax), small against
    the overlap's rate, so that contacts hold, stick and slide from the
    start.  k_n = k_t = k, mu_s = mu_d = mu, dt = 5e-7 s, gravity -9.81
    m/s^2.  gamma_n is gamma_frac of critical: contact model 2's normal
    viscosity feeds a vibrating packing (see ``packed``), slowly at this
    value."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    m = 2600.0 * float(V_sphere(r))
    s0 = 2.0 * r
    delta = sigma * s0 * s0 / k
    spacing = s0 - delta
    sb = Spherebin(np_=n, nw=0, sid=sid)
    idx = np.arange(n)
    lat = np.stack([idx % nx, (idx // nx) % ny, idx // (nx * ny)], axis=1).astype(float)
    sb.x = lat * spacing + (r - delta)
    sb.x += rng.uniform(-0.01 * delta, 0.01 * delta, size=(n, 3))
    sb.radius = np.full(n, r)
    sb.vel = rng.uniform(-vmax, vmax, size=(n, 3))
    sb.angvel = rng.uniform(-wmax, wmax, size=(n, 3))
    sb.origo = np.zeros(3)
    sb.L = np.array([nx, ny, nz], dtype=float) * spacing - spacing + 2.0 * (r - delta)
    sb.num = np.floor(sb.L / (2.2 * r)).astype(np.uint32)
    sb.periodic = 0
    sb.g = np.array([0.0, 0.0, -9.81])
    gamma = gamma_frac * 2.0 * math.sqrt(k * m)
    _contact_params(sb, k_n=k, k_t=k, gamma_n=gamma, gamma_t=0.0, mu=mu, gamma_w=gamma)
    sb.time_dt = dt
    sb.time_total = 4000 * dt
    sb.time_file_dt = sb.time_total
    return sb


def ensemble(n_inst=512, cell_factor=2.0, first=0):
    """The batched settling ensemble: members first .. first + n_inst - 1."""
    return [ensemble_member(first + i, cell_factor=cell_factor) for i in range(n_inst)]


def column(n=100_000, seed=0, col=(0.1, 0.1, 0.3), box=(0.6, 0.6, 0.35), k=1e6, mu=0.5,
           dt=5e-7, sid="column") -> Spherebin:
    """The calibration column: n spheres with the radii of ``polydisperse``
    (log-normal, median 1 mm, sigma 0.2, clipped 0.5-2 mm), placed by random
    sequential placement in a col[0] x col[1] x col[2] column standing on the
    floor at the centre of a non-periodic box with the implicit frictional
    walls; gravity -9.81 m/s^2, k_n = k_t = k, mu_s = mu_d = mu (walls too),
    dt = 5e-7 s.  gamma_n (and the wall damping) is 0.48 of the critical
    2 sqrt(m k_n) at the 1 mm mass, the damping ratio of ``settling``: the
    settling scene's 100 N s/m would damp a millimetre grain by a factor
    gamma dt / m of about 5 per step, which the explicit step cannot
    integrate.  Cells are 2 r_max wide."""
    rng = np.random.default_rng(seed)
    radii = _lognormal_radii(rng, n)
    pos = rsa_place(rng, radii, col, periodic_xy=False)
    box = np.asarray(box, float)
    pos[:, 0] += 0.5 * (box[0] - col[0])
    pos[:, 1] += 0.5 * (box[1] - col[1])
    sb = Spherebin(np_=n, nw=0, sid=sid)
    sb.radius = radii
    sb.x = pos
    sb.origo = np.zeros(3)
    sb.L = box
    sb.num = np.floor(box / (2.0 * float(radii.max()))).astype(np.uint32)
    sb.periodic = 0
    sb.g = np.array([0.0, 0.0, -9.81])
    m_ref = 4.0 / 3.0 * math.pi * 1e-3 ** 3 * 2600.0
    gamma_n = 0.48 * 2.0 * math.sqrt(m_ref * k)
    _contact_params(sb, k_n=k, k_t=k, gamma_n=gamma_n, gamma_t=0.0, mu=mu, gamma_w=gamma_n)
    sb.time_dt = dt
    sb.time_total = 4000 * dt
    sb.time_file_dt = sb.time_total
    return sb
