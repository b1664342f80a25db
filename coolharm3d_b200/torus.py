"""Fishbone-Moncrief torus around a Kerr black hole: grid description and
initial data of the reference's torus setup (init.torus.c), the problem the
engine's throughput is quoted on.

The grid is modified Kerr-Schild (COORD_DIAGONAL3) with spherical outflow-3
boundaries, PPM_MC reconstruction, HLLE fluxes, parabolic flux-CT, the entropy
fix, RESCALE_R and H/R disk cooling.  The initial data restates the
published Fishbone & Moncrief (1976) solution as init_prim() evaluates it
(init.torus.c:355-474), normalised to rho_max = 1, with the poloidal field of
set_mag_field() (init.torus.c:489-585): A_phi = max(rho_avg - 0.2, 0) at zone
corners, B by central differences of A_phi, scaled to plasma beta 100.

The setup drives a target with the methods upload(p), fixup_bounds() and
download() -- an Engine, whose floors and boundary kernels are the ones the
step uses -- the way init_data() interleaves its analytic fields with
fixup(p); bounds(p,0) (init.torus.c:172-216).

The reference perturbs u by randfact * (ranc() - 0.5) with ranc() seeded from
the wall clock (ranc.c:37-41), so its perturbation is not reproducible; here
the perturbation is drawn from numpy's PCG64 with an explicit seed.
"""
import math

import numpy as np

from . import (BC_SPHERICAL_OUTFLOW3, FLUX_HLLE, NG, PREC_FP64, RECON_PPM_MC, ks_mks_tables, make_desc,
               ref_shape)

SMALL = 1.0e-15         # macros.h:441
RHOMIN = 2.0e-10        # options.h:233
UUMIN = 2.0e-12         # options.h:234
CENT = 3                # geometry position of the zone centre (macros.h:187)
G_GCON, G_GCOV, G_G, G_BETA, G_NCON = 0, 16, 32, 35, 38


def horizon_radius(a):
    """Outer horizon r_+ = 1 + sqrt(1 - a^2) (rhorizon_calc, metric.c:504-511)."""
    return 1.0 + math.sqrt((1.0 - a) * (1.0 + a))


def inner_radius(n1, a, r_out, r0=0.0, n_within_horizon=5):
    """Inner radial edge that puts the horizon n_within_horizon - 1/4 zones
    inside the grid on a logarithmic radial grid (Rin_calc, coord.c:2556-2571)."""
    fn = n_within_horizon - 0.25
    x0 = (n1 * math.log(horizon_radius(a) - SMALL - r0) - fn * math.log(r_out - r0)) / (n1 - fn)
    return r0 + math.exp(x0)


def torus_desc(n, a=0.9, r_out=120.0, r0=0.0, n_within_horizon=5, gam=5.0 / 3.0, cour=0.8, dt0=1.0e-5,
               t_final=1.0e4, phi_length=2.0 * math.pi, precision=PREC_FP64, device=0):
    """GridDesc of the torus run on n = (N1, N2, N3) zones (init_base,
    init.torus.c:55-104): x1 = log(r - R0) over [log(Rin - R0), log(Rout - R0)],
    x2 over [0, 1], x3 = phi over [0, phi_length]."""
    n1, n2, n3 = (int(x) for x in n)
    r_in = inner_radius(n1, a, r_out, r0, n_within_horizon)
    length = [t_final, math.log((r_out - r0) / (r_in - r0)), 1.0, phi_length]
    dx = [dt0, length[1] / n1, length[2] / n2, length[3] / n3]
    startx = [0.0, math.log(r_in - r0) - NG * dx[1], 0.0 - NG * dx[2], 0.0 - NG * dx[3]]
    return make_desc((n1, n2, n3), gam, cour, dx, startx, length, recon=RECON_PPM_MC, flux=FLUX_HLLE, ct_para=1,
                     bc=BC_SPHERICAL_OUTFLOW3, metric_dim=2, use_ee=1, cooling=1, rescale_r=1, precision=precision,
                     device=device)


def torus_tables(desc, a=0.9, h_o_r=0.1):
    """Geometry, per-zone data and cooling tables of the torus grid."""
    return ks_mks_tables(desc, a, R0=0.0, h_slope=0.35, th_cutout=SMALL * math.pi, diag3_exponent=7, h_o_r=h_o_r)


def angular_momentum(r, a, prograde=True):
    """u_phi u^t of the circular orbit at r, constant through the torus
    (lfish_calc2, init.torus.c:596-621)."""
    s = 1.0 if prograde else -1.0
    sr = math.sqrt(r)
    rsq, asq = r * r, a * a
    return s * (rsq * (rsq + asq) - 2 * r * asq - s * a * sr * (rsq - asq)) / (sr * r * (rsq - 3.0 * r + 2.0 * s * a * sr))


def _geom_cent(tables, n1t, n2t):
    g = np.asarray(tables["geom"]).reshape(5, n1t, n2t, 42)
    return g[CENT]


def hydro_fields(desc, tables, a=0.9, r_in=6.0, r_max=12.0, kappa=1.0e-3):
    """Axisymmetric torus fields on the physical (i, j) zones: rho, u (before
    normalisation and perturbation), the numerical-frame velocity primitives
    U1..U3, a mask of the zones inside the torus, and rho_max, u_max
    (init_prim, init.torus.c:355-474)."""
    gam = desc.gam
    n1, n2 = desc.n1, desc.n2
    n1t, n2t, _ = ref_shape((desc.n1, desc.n2, desc.n3))
    c6 = np.asarray(tables["cell6"])
    r = c6[NG:NG + n1, NG:NG + n2, NG, 2]
    th = c6[NG:NG + n1, NG:NG + n2, NG, 4]
    sth, cth = np.sin(th), np.cos(th)
    l = angular_momentum(r_max, a)

    DD = r * r - 2.0 * r + a * a
    AA = (r * r + a * a) * (r * r + a * a) - DD * a * a * sth * sth
    SS = r * r + a * a * cth * cth
    DDin = r_in * r_in - 2.0 * r_in + a * a
    AAin = (r_in * r_in + a * a) * (r_in * r_in + a * a) - DDin * a * a
    SSin = r_in * r_in
    with np.errstate(invalid="ignore", divide="ignore"):
        lnh_in = (0.5 * math.log((1.0 + math.sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin / (AAin * AAin)))
                                 / (SSin * DDin / AAin))
                  - 0.5 * math.sqrt(1.0 + 4.0 * (l * l * SSin * SSin) * DDin / (AAin * AAin))
                  - 2.0 * a * r_in * l / AAin)
        lnh = (0.5 * np.log((1.0 + np.sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD / (AA * sth * AA * sth)))
                            / (SS * DD / AA))
               - 0.5 * np.sqrt(1.0 + 4.0 * (l * l * SS * SS) * DD / (AA * AA * sth * sth))
               - 2.0 * a * r * l / AA
               - lnh_in)
        lnh = np.where(r >= r_in, lnh, 1.0)
        inside = ~((lnh < 0.0) | (r < r_in))

        hm1 = np.exp(lnh) - 1.0
        rho = np.where(inside, np.power(np.where(inside, hm1, 1.0) * (gam - 1.0) / (kappa * gam), 1.0 / (gam - 1.0)),
                       -RHOMIN * 1.0e-14)
        u = np.where(inside, kappa * np.power(np.abs(rho), gam) / (gam - 1.0), UUMIN * 1.0e-14)

        # u^phi of the Boyer-Lindquist orbit, then u^t from u.u = -1 with the
        # BL metric (setutcon, metric.c:78-101); u^r = u^th = 0, so the
        # BL -> KS map (metric.c:1940-1954) and the diagonal KS -> MKS
        # Jacobian leave (u^t, 0, 0, u^phi) as it is
        expm2chi = SS * SS * DD / (AA * AA * sth * sth)
        up1 = np.sqrt((-1.0 + np.sqrt(1.0 + 4.0 * l * l * expm2chi)) / 2.0)
        up = 2.0 * a * r * np.sqrt(1.0 + up1 * up1) / np.sqrt(AA * SS * DD) + np.sqrt(SS / AA) * up1 / sth
        sig = r * r + a * a * cth * cth
        s2 = sth * sth
        g_tt = -1.0 + 2.0 * r / sig
        g_tp = -2.0 * a * r * s2 / sig
        g_pp = (r * r + a * a + 2.0 * a * a * r * s2 / sig) * s2
        b = g_tp * up
        c = g_pp * up * up + 1.0
        ut = (-b - np.sqrt(b * b - g_tt * c)) / g_tt

    # ucon2pr (phys.c:302-312) with the MKS inverse metric at the zone centre
    gc = _geom_cent(tables, n1t, n2t)[NG:NG + n1, NG:NG + n2]
    f = ut / gc[..., G_GCON + 0]
    vel = np.zeros((n1, n2, 3))
    vel[..., 0] = 0.0 - gc[..., G_GCON + 1] * f
    vel[..., 1] = 0.0 - gc[..., G_GCON + 2] * f
    vel[..., 2] = up - gc[..., G_GCON + 3] * f
    vel[~inside] = 0.0
    rho_max = float(rho[inside].max())
    u_max = float(u[inside & (r > r_in)].max())
    return dict(rho=rho, u=u, vel=vel, inside=inside, rho_max=rho_max, u_max=u_max)


def _bsq(p_ij, geom_ij):
    """b^mu b_mu of the primitives p_ij[..., 8] (bsq_calc, phys.c:190-214)."""
    gcov = geom_ij[..., G_GCOV:G_GCOV + 16].reshape(geom_ij.shape[:-1] + (4, 4))
    v = p_ij[..., 2:5]
    qsq = np.einsum("...a,...ab,...b->...", v, gcov[..., 1:, 1:], v)
    gamma = np.sqrt(1.0 + qsq)
    ucon = np.empty(p_ij.shape[:-1] + (4,))
    ucon[..., 0] = gamma * geom_ij[..., G_NCON]
    ucon[..., 1:] = v - ucon[..., :1] * geom_ij[..., G_BETA:G_BETA + 3]
    ucov = np.einsum("...ab,...b->...a", gcov, ucon)
    B = p_ij[..., 5:8]
    bcon = np.empty_like(ucon)
    bcon[..., 0] = np.einsum("...a,...a->...", B, ucov[..., 1:])
    bcon[..., 1:] = (B + bcon[..., :1] * ucon[..., 1:]) / ucon[..., :1]
    return np.einsum("...a,...ab,...b->...", bcon, gcov, bcon)


def set_torus(target, desc, tables, a=0.9, r_in=6.0, r_max=12.0, kappa=1.0e-3, beta=100.0, randfact=4.0e-2,
              seed=12345, return_prims=True):
    """Initial data of the magnetised torus on `target` (init_data,
    init.torus.c:172-216).  Returns the final primitives in the reference
    layout when return_prims, else None (they stay resident in the target)."""
    n1, n2, n3 = desc.n1, desc.n2, desc.n3
    shp = ref_shape((n1, n2, n3))
    h = hydro_fields(desc, tables, a, r_in, r_max, kappa)
    rho_max = h["rho_max"]
    u_max = h["u_max"] / rho_max

    p = np.zeros(shp + (8,))
    phys = (slice(NG, NG + n1), slice(NG, NG + n2), slice(NG, NG + n3))
    pert = np.ones((n1, n2, n3))
    if randfact:
        rng = np.random.Generator(np.random.PCG64(seed))
        pert = 1.0 + randfact * (rng.random((n1, n2, n3)) - 0.5)
        pert[~h["inside"]] = 1.0
    p[phys + (0,)] = (h["rho"] / rho_max)[:, :, None]
    p[phys + (1,)] = h["u"][:, :, None] * pert / rho_max
    p[phys + (slice(2, 5),)] = h["vel"][:, :, None, :]
    target.upload(p)
    target.fixup_bounds()
    p = target.download()

    # A_phi at the corners (i, j) = N1S..N1E+1, N2S..N2E+1 from rho in the
    # k = N3S slice; rho_max is 1 after the normalisation
    rk = p[:, :, NG, 0]
    i0, i1, j0, j1 = NG, NG + n1 + 1, NG, NG + n2 + 1
    rho_avg = 0.25 * (rk[i0:i1, j0:j1] + rk[i0 - 1:i1 - 1, j0:j1] + rk[i0:i1, j0 - 1:j1 - 1] +
                      rk[i0 - 1:i1 - 1, j0 - 1:j1 - 1])
    q = rho_avg / 1.0 - 0.2
    A = np.where(q > 0.0, q, 0.0)
    gc = _geom_cent(tables, shp[0], shp[1])[NG:NG + n1, NG:NG + n2]
    gdet = gc[..., G_G]
    B = np.zeros((n1, n2, 3))
    B[..., 0] = -(A[:-1, :-1] - A[:-1, 1:] + A[1:, :-1] - A[1:, 1:]) / (2.0 * desc.dx[2] * gdet)
    B[..., 1] = (A[:-1, :-1] + A[:-1, 1:] - A[1:, :-1] - A[1:, 1:]) / (2.0 * desc.dx[1] * gdet)
    # bsq with the velocities of the k = 0 slice, as set_mag_field reads them
    pk = p[NG:NG + n1, NG:NG + n2, 0].copy()
    pk[..., 5:8] = B
    bsq_max = float(_bsq(pk, gc).max())
    beta_act = (desc.gam - 1.0) * u_max / (0.5 * bsq_max)
    norm = math.sqrt(beta_act / beta)
    B[..., 0] *= norm
    B[..., 1] *= norm
    p[..., 5:8] = 0.0
    p[NG:NG + n1, NG:NG + n2, :, 5:8] = B[:, :, None, :]
    target.upload(p)
    target.fixup_bounds()
    return target.download() if return_prims else None
