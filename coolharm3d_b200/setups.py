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


def _minkowski_u_f(P, gam):
    """HARM's conserved variables and its three directional fluxes of ideal
    MHD in Minkowski space for one primitive state P = (rho, u, u~1..3,
    B1..3): ucon_calc / bcon_calc (phys.c:216, 75) with alpha 1, beta 0;
    mhd_calc (phys.c:93) T^mu_nu = w u^mu u_nu + p_tot delta - b^mu b_nu;
    primtoflux (phys.c:28): rho u^mu, T^mu_t + rho u^mu, T^mu_j,
    b^j u^mu - b^mu u^j (B^j itself for mu = t).  Works on complex P, for
    complex-step derivatives."""
    rho, u, v1, v2, v3, B1, B2, B3 = P
    ut = np.sqrt(1.0 + v1 * v1 + v2 * v2 + v3 * v3)
    ucon = [ut, v1, v2, v3]
    bt = B1 * v1 + B2 * v2 + B3 * v3
    bcon = [bt] + [(Bj + bt * ucon[j + 1]) / ut for j, Bj in enumerate((B1, B2, B3))]
    sgn = (-1.0, 1.0, 1.0, 1.0)
    ucov = [sgn[m] * ucon[m] for m in range(4)]
    bcov = [sgn[m] * bcon[m] for m in range(4)]
    bsq = sum(bcon[m] * bcov[m] for m in range(4))
    pg = (gam - 1.0) * u
    w, ptot = rho + u + pg + bsq, pg + 0.5 * bsq

    def row(mu):
        T = [w * ucon[mu] * ucov[nu] + (ptot if mu == nu else 0.0) - bcon[mu] * bcov[nu] for nu in range(4)]
        out = [rho * ucon[mu], T[0] + rho * ucon[mu], T[1], T[2], T[3]]
        out += [B1, B2, B3] if mu == 0 else [bcon[j] * ucon[mu] - bcon[mu] * ucon[j] for j in (1, 2, 3)]
        return np.array(out)

    return row(0), [row(1), row(2), row(3)]


def rmhd_modes(rho, pgas, gam, B, nhat):
    """Linear eigenmodes of relativistic ideal MHD about the static state
    (rho, p, v = 0, B) for plane waves along nhat: the eigenvalues lambda
    (wave speeds, ascending: fast-, Alfven-, slow-, entropy, slow+, Alfven+,
    fast+) and primitive right eigenvectors R (8 x 7, columns in the same
    order) of  n_d dF^d/dP R = lambda dU/dP R  with dB.nhat = 0.  The
    Jacobians are complex-step derivatives of _minkowski_u_f; the perturbed
    field is restricted to the plane normal to nhat and the equations
    projected on it, which drops the zero-speed divergence mode.  The
    reference's closed forms (eigs(), init.linearwave.c:166-240, for
    B = (Bx, 0, 0) along k = 2 pi (1, 1, 0)) are special cases."""
    nhat = np.asarray(nhat, float) / np.linalg.norm(nhat)
    P = np.array([rho, pgas / (gam - 1.0), 0.0, 0.0, 0.0, *B], float)
    h = 1.0e-30
    dU, dF = np.zeros((8, 8)), np.zeros((8, 8))
    for c in range(8):
        Pc = P.astype(complex)
        Pc[c] += 1j * h
        U, F = _minkowski_u_f(Pc, gam)
        dU[:, c] = U.imag / h
        dF[:, c] = sum(nhat[d] * F[d].imag for d in range(3)) / h
    a = np.array([1.0, 0.0, 0.0]) if abs(nhat[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = a - nhat * np.dot(a, nhat)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(nhat, e1)
    Q = np.zeros((8, 7))
    Q[:5, :5] = np.eye(5)
    Q[5:, 5], Q[5:, 6] = e1, e2
    A = np.linalg.solve(Q.T @ dU @ Q, Q.T @ dF @ Q)
    lam, V = np.linalg.eig(A)
    if np.abs(lam.imag).max() > 1e-12 or np.abs(V.imag).max() > 1e-12:
        raise ValueError("complex eigenmodes: the background state is not hyperbolic")
    o = np.argsort(lam.real)
    return lam.real[o], Q @ V.real[:, o]


MODES = {"fast": 6, "alfven": 5, "slow": 4}


def eigenmode(mode, rho, pgas, gam, B, nhat):
    """One right-moving mode ('fast', 'alfven' or 'slow') of rmhd_modes:
    (dp, lambda), dp scaled so that its largest component is +1.  Raises
    ValueError if the mode's speed is degenerate with a neighbour's (field
    along nhat or normal to it), where the eigenvector is not unique."""
    lam, R = rmhd_modes(rho, pgas, gam, B, nhat)
    m = MODES[mode]
    gap = min(abs(lam[m] - lam[m - 1]), abs(lam[m + 1] - lam[m]) if m < 6 else np.inf)
    if gap < 1e-8:
        raise ValueError("%s mode is degenerate for this field direction" % mode)
    dp = R[:, m] / R[np.argmax(np.abs(R[:, m])), m]
    dp[np.abs(dp) < 1e-14] = 0.0
    return dp, float(lam[m])


def linear_wave_3d(n, mode="fast", amp=1.0e-6, rho=1.0, pgas=1.0, gam=4.0 / 3.0, B=(1.0, 1.5, 0.0), kvec=(1, 1, 1),
                   cour=0.4, recon=RECON_PPM_MC, precision=PREC_FP64, device=0):
    """Periodic linear wave of one exact RMHD eigenmode on the unit box:
    p = p0 + amp dp cos(k.x), k = 2 pi kvec (integers, so the box holds
    whole wavelengths), with (dp, lambda) from eigenmode along kvec; one
    period is t_f = 2 pi / (|k| lambda), after which the exact solution is
    the initial state again.  The default is the fast mode of rho 1, p 1,
    B (1, 1.5, 0), Gamma 4/3 along the grid diagonal at amplitude 1e-6;
    PPM_MC (or `recon`) + HLLE + para flux-CT like the reference's
    linear-wave test (init.linearwave.c).  With n3 = 1, kvec must have no x3
    component."""
    n = tuple(int(x) for x in n)
    kvec = np.asarray(kvec, float)
    if n[2] == 1 and kvec[2] != 0:
        raise ValueError("a grid with one zone in x3 cannot hold a wave with k3 != 0")
    dp, lam = eigenmode(mode, rho, pgas, gam, B, kvec)
    k = 2.0 * math.pi * kvec
    tf = 2.0 * math.pi / (np.linalg.norm(k) * lam)
    dx = [1.0e-5] + [1.0 / x for x in n]
    startx = [0.0] + [0.0 - NG * dx[a] for a in (1, 2, 3)]
    desc = make_desc(n, gam, cour, dx, startx, [tf, 1.0, 1.0, 1.0], recon=recon, flux=FLUX_HLLE, ct_para=1,
                     bc=BC_CARTESIAN_PERIODIC, metric_dim=0, use_ee=1, precision=precision, device=device)
    shp = ref_shape(n)
    x1, x2, x3 = (_centres(desc, a) for a in (1, 2, 3))
    eph = np.cos(k[0] * x1[:, None, None] + k[1] * x2[None, :, None] + k[2] * x3[None, None, :])
    base = np.array([rho, pgas / (gam - 1.0), 0.0, 0.0, 0.0, *B])
    p = np.zeros(shp + (8,))
    sl = tuple(slice(NG, NG + x) for x in n)
    for l in range(8):
        p[sl + (l,)] = (base[l] + dp[l] * amp * eph)[sl]
    return _problem("linear_wave_3d_" + mode, desc, p, tf)


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
