"""Minkowski problem setups of the reference (init.balsara1.c,
init.linearwave.c, init.field_loop.c): grid description, geometry and floor
tables, initial primitives and final time, restated from those files.

Each setup returns a Problem.  `start(target, problem)` loads it into a
target with the Engine methods set_geometry / set_cell_data / upload /
fixup_bounds / set_time, the way each init_data() ends with
fixup(p); bounds(p,0).
"""
import math
from dataclasses import dataclass

import numpy as np

from . import (BC_CARTESIAN_OUTFLOW, BC_CARTESIAN_PERIODIC, FLUX_HLLE, NG, PREC_FP64, RECON_MC, RECON_PPM_MC,
               make_desc, minkowski_tables, ref_shape)


@dataclass
class Problem:
    name: str
    desc: object          # GridDesc
    geom: np.ndarray      # one struct of_geom (Minkowski)
    cell6: np.ndarray     # per-zone floors and coordinates
    p_init: np.ndarray    # primitives before fixup/bounds, reference layout
    t_final: float

    @property
    def n(self):
        return (self.desc.n1, self.desc.n2, self.desc.n3)

    @property
    def zones(self):
        return self.desc.n1 * self.desc.n2 * self.desc.n3


def _centres(desc, a):
    """Zone-centre coordinates x^a of every reference index (ghosts included)."""
    n = (desc.n1, desc.n2, desc.n3)[a - 1]
    return desc.startx[a] + (np.arange(n + 2 * NG) + 0.5) * desc.dx[a]


def _problem(name, desc, p, t_final):
    geom, cell6 = minkowski_tables(desc)
    return Problem(name, desc, geom, cell6, p, t_final)


def balsara1(n1, cour=0.5, recon=RECON_MC, flux=FLUX_HLLE, ct_para=1, use_ee=1, precision=PREC_FP64, device=0):
    """Balsara test 1 shock tube on x in [-0.5, 0.5], Gamma 2, to t = 0.4
    (init.balsara1.c): left rho 1, p 1, B (0.5, 1, 0); right rho 0.125,
    p 0.1, B (0.5, -1, 0); outflow boundaries.  The reference ships
    cour 0.8; the benchmark configuration uses 0.5."""
    n = (int(n1), 1, 1)
    gam = 2.0
    dx = [1.0e-5, 1.0 / n[0], 1.0, 1.0]
    startx = [0.0] + [-0.5 - NG * dx[a] for a in (1, 2, 3)]
    desc = make_desc(n, gam, cour, dx, startx, [0.4, 1.0, 1.0, 1.0], recon=recon, flux=flux, ct_para=ct_para,
                     bc=BC_CARTESIAN_OUTFLOW, metric_dim=0, use_ee=use_ee, precision=precision, device=device)
    shp = ref_shape(n)
    p = np.zeros(shp + (8,))
    left = _centres(desc, 1) < 0.0
    phys = np.zeros(shp[0], bool)
    phys[NG:NG + n[0]] = True
    L, R = phys & left, phys & ~left
    p[L, :, :, 0], p[L, :, :, 1], p[L, :, :, 5], p[L, :, :, 6] = 1.0, 1.0 / (gam - 1.0), 0.5, 1.0
    p[R, :, :, 0], p[R, :, :, 1], p[R, :, :, 5], p[R, :, :, 6] = 0.125, 0.1 / (gam - 1.0), 0.5, -1.0
    # a degenerate direction is all one zone: the reference fills only the
    # physical index there too (LOOP), and the boundaries copy it
    mask = np.zeros(shp, bool)
    mask[NG:NG + n[0], NG:NG + 1, NG:NG + 1] = True
    p[~mask] = 0.0
    return _problem("balsara1", desc, p, 0.4)


def slow_mode(Bx):
    """Eigenvector and frequency of the slow magnetosonic mode of the
    reference's linear-wave test (eigs(), init.linearwave.c, SLOW branch):
    rho0 = 1, u0 = 1/(Gamma - 1) with Gamma 4/3, B0 = (Bx, 0, 0), k = 2 pi (1, 1, 0)."""
    Bx2 = Bx * Bx
    aux1 = 400.0 + 80.0 * Bx2 + 169.0 * Bx2 * Bx2
    r1 = 2.0 * math.pi * math.sqrt((20.0 + 17.0 * Bx2 - math.sqrt(aux1)) / (75.0 + 15.0 * Bx2))
    r2 = 2.0 * math.pi * math.sqrt((20.0 + 17.0 * Bx2 + math.sqrt(aux1)) / (75.0 + 15.0 * Bx2))
    dp = np.zeros(8)
    s = 1.0 if r2 > r1 else -1.0    # the root of the slower branch
    dp[0] = (-20.0 + 13 * Bx2 + s * math.sqrt(aux1)) / 20.0
    dp[1] = (-20.0 + 13 * Bx2 + s * math.sqrt(aux1)) / 5.0
    dp[2] = math.sqrt((20.0 + 17.0 * Bx2 - s * math.sqrt(aux1)) / (75.0 + 15.0 * Bx2)) * \
        (13.0 * Bx2 + s * math.sqrt(aux1)) / 20.0
    dp[3] = -math.sqrt((20.0 + 17.0 * Bx2 - s * math.sqrt(aux1)) / (75.0 + 15.0 * Bx2))
    dp[5] = -Bx
    dp[6] = Bx
    return dp, (r1 if r2 > r1 else r2)


def linear_wave(n, amp=1.0e-4, cour=0.4, precision=PREC_FP64, device=0):
    """The reference's periodic linear-wave test (init.linearwave.c): the slow
    mode above on the unit box (any N3; the wave does not depend on x3),
    PPM_MC + HLLE + para flux-CT, run for one wave period 2 pi / w."""
    n = tuple(int(x) for x in n)
    gam = 4.0 / 3.0
    dx = [1.0e-5] + [1.0 / x for x in n]
    startx = [0.0] + [0.0 - NG * dx[a] for a in (1, 2, 3)]
    dp, w = slow_mode(1.0)
    tf = 2.0 * math.pi / w
    desc = make_desc(n, gam, cour, dx, startx, [tf, 1.0, 1.0, 1.0], recon=RECON_PPM_MC, flux=FLUX_HLLE, ct_para=1,
                     bc=BC_CARTESIAN_PERIODIC, metric_dim=0, use_ee=1, precision=precision, device=device)
    shp = ref_shape(n)
    x1, x2 = _centres(desc, 1), _centres(desc, 2)
    eph = np.cos(2.0 * math.pi * x1[:, None] + 2.0 * math.pi * x2[None, :])
    base = np.array([1.0, 1.0 / (gam - 1.0), 0, 0, 0, 1.0, 0, 0])
    p = np.zeros(shp + (8,))
    sl = tuple(slice(NG, NG + x) for x in n)
    for l in range(8):
        p[sl + (l,)] = (base[l] + dp[l] * amp * eph)[sl[0], sl[1], None]
    return _problem("linear_wave", desc, p, tf)


def field_loop(n, v0=0.5, loop_radius=0.3, az0=1.0e-3, cour=0.4, precision=PREC_FP64, device=0):
    """Advected magnetic field loop (init.field_loop.c; Gardiner & Stone 2005)
    on [-3, 3]^2, periodic, Gamma 5/3, rho 1, p 3, v = (v0, v0/2, 0), to
    t = 25 (10 if v0 = 0).  A_z = Az0 (R - r) inside the loop radius R,
    r measured in the loop's rest frame, and B = curl A with the four-edge
    averages of curl_of_A (flux_ct.c:996-1066).

    The reference builds A_mu with a Lorentz matrix whose (z, y) entry is
    never assigned (init.field_loop.c sets (y, z) twice); for v_z = 0 the
    value it stands for is 0, which is used here."""
    n = tuple(int(x) for x in n)
    gam = 5.0 / 3.0
    dx1, dx2 = 6.0 / n[0], 6.0 / n[1]
    dx3 = dx2
    dx = [1.0e-5, dx1, dx2, dx3]
    startx = [0.0, -3.0 - NG * dx1, -3.0 - NG * dx2, -0.5 * dx3 - NG * dx3]
    t_final = 25.0 if v0 >= 1e-15 else 10.0
    desc = make_desc(n, gam, cour, dx, startx, [t_final, 6.0, 6.0, n[2] * dx3], recon=RECON_PPM_MC, flux=FLUX_HLLE,
                     ct_para=1, bc=BC_CARTESIAN_PERIODIC, metric_dim=0, use_ee=1, precision=precision, device=device)
    shp = ref_shape(n)
    vx, vy = v0, 0.5 * v0
    gamma = 1.0 / math.sqrt(1.0 - vx * vx - vy * vy)
    p = np.zeros(shp + (8,))
    sl = tuple(slice(NG, NG + x) for x in n)
    p[sl + (0,)] = 1.0
    p[sl + (1,)] = 3.0 / (gam - 1.0)
    p[sl + (2,)] = gamma * vx
    p[sl + (3,)] = gamma * vy
    # A_z at the zone corners (i, j) = N1S..N1E+1, N2S..N2E+1, in the rest
    # frame of the loop: (x', y') = Lambda (x, y), Lambda the boost by -v
    # built from v recovered from u^mu as set_mag_field does
    g4 = gamma
    vxr, vyr = (g4 * vx) / g4, (g4 * vy) / g4
    v2 = vxr * vxr + vyr * vyr + 0.0 * 0.0
    if v2 > 0:
        Lxx = 1.0 + (g4 - 1.0) * vxr * vxr / v2
        Lyy = 1.0 + (g4 - 1.0) * vyr * vyr / v2
        Lxy = (g4 - 1.0) * vxr * vyr / v2
    else:
        Lxx, Lyy, Lxy = 1.0, 1.0, 0.0
    xc = desc.startx[1] + np.arange(NG, NG + n[0] + 1) * dx1
    yc = desc.startx[2] + np.arange(NG, NG + n[1] + 1) * dx2
    X, Y = np.meshgrid(xc, yc, indexing="ij")
    xr = X * Lxx + Y * Lxy
    yr = X * Lxy + Y * Lyy
    r = np.sqrt(xr * xr + yr * yr)
    Az = np.where(r <= loop_radius, az0 * (loop_radius - r), 0.0)
    f1, f2 = 0.25 * (1.0 / dx1), 0.25 * (1.0 / dx2)
    # curl_of_A's four-edge sums, left to right; A does not depend on x3, so
    # the k+1 edges repeat the k edges
    a00, a01, a10, a11 = Az[:-1, :-1], Az[:-1, 1:], Az[1:, :-1], Az[1:, 1:]
    s1 = a01 - a00 + a11 - a10 + a01 - a00 + a11 - a10
    s2 = a10 - a00 + a11 - a01 + a10 - a00 + a11 - a01
    b1 = f2 * s1 - 0.0
    b2 = 0.0 - f1 * s2
    p[sl + (5,)] = b1[:, :, None]
    p[sl + (6,)] = b2[:, :, None]
    return _problem("field_loop", desc, p, t_final)


def start(target, problem, t=0.0):
    """Load the problem into the target: tables, initial primitives, the
    setups' closing fixup(p); bounds(p,0), and the first time step."""
    target.set_geometry(problem.geom)
    target.set_cell_data(problem.cell6)
    target.upload(problem.p_init)
    target.fixup_bounds()
    target.set_time(t, problem.desc.dx[0])
