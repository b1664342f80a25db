"""Circumbinary disk around an equal-mass black-hole binary: grid
description and initial data of the reference's post-Newtonian binary disk
setup (init.nz_pn_bbh_disk.c), the configuration whose metric changes in
time and is evaluated on the device every substep (metric_dim 3).

The binary: masses 0.5 + 0.5 (M = 1), separation 20M, no spins
(set_special_coord, init.nz_pn_bbh_disk.c:308-350).  The grid is
COORD_DIAGONAL3 spherical, x1 = log(r - R0) over [Rin, Rout], x2 over [0, 1]
with the focusing h_slope = 0.0729419909586 and diag3_exponent 9, x3 = phi
over [0, 2 pi]; spherical outflow-3 boundaries, PPM_MC + HLLE, parabolic
flux-CT, the entropy fix, RESCALE_R and H/R = 0.1 disk cooling.  The run's
parameters put r over [0.75a, 13a] and the loop's plasma beta at 10 (the
shipped file: [0.05a, 100a], beta 100).

The disk is De Villiers, Hawley & Krolik's power-law torus (q = 1.58,
Keplerian l(Omega)) about a Schwarzschild mass M in Boyer-Lindquist
coordinates, r_BL = r + M, inner edge 2(a + M), pressure maximum 5(a + M),
K = 0.01 polytrope, u perturbed by 1% with the reference's ranc() seeded
with 1 (init_prim, rho_func, find_l_ang_in, get_rpmax, find_l_bracket:
init.nz_pn_bbh_disk.c:405-533, 668-974).  Its 4-velocity (u^t, 0, 0, u^phi)
becomes primitives through the grid metric's gcon (ucon2pr, phys.c:302-312),
and the poloidal field follows the density (set_mag_field,
init.nz_pn_bbh_disk.c:535-660): A_phi = max(rho_avg - rho_max/4, 0) at zone
corners of the k = N3S slice, B by differences of A_phi with sqrt(-g) of the
k = 0 layer, scaled so that the integrated plasma beta is 10.

The scalar parts (the l bracket and bisections, the BL metric, rho_func) run
in Python floats in the reference's operation order with the platform's libm,
so they reproduce the reference's doubles; the grid-wide steps are numpy in
the same order.  ranc() is restated from its algorithm (ranc.c): 64
multiplicative lanes seeded from the C library's rand() after srand(seed).

The shipped setup moves the grid's stored coordinate x[RR] of every zone to
the Boyer-Lindquist radius in place and moves it back only inside the disk
(init.nz_pn_bbh_disk.c:494-507); the reference's run would then evaluate its
metric, RESCALE_R and cooling tables at r + M outside the disk.  This setup
leaves the grid's coordinates as they are (the reference configuration it
is checked against restores them), so its tables are the grid's own.
"""
import copy
import ctypes
import ctypes.util
import math

import numpy as np

from . import (BC_SPHERICAL_OUTFLOW3, FLUX_HLLE, NG, PREC_FP64, RECON_PPM_MC, dyn_metric, ks_mks_tables, make_desc,
               ref_shape)

SMALL = 1.0e-15          # macros.h:441
SINGSMALL = 1.0e-16      # options.h:271
M_BH1 = M_BH2 = 0.5
M_TOT = M_BH1 + M_BH2
SPIN = 0.0
SEPARATION = 20.0 * M_TOT
H_SLOPE = 0.0729419909586
DIAG3_EXPONENT = 9
TH_CUTOUT = math.pi * SMALL
L_ANG_PRECISION = 1.0e-6
R_DISK_MAX = 1.0e6
L_DISK_MAX = 1.0e4
CENT = 3
G_GCON, G_GCOV, G_G, G_BETA, G_NCON = 0, 16, 32, 35, 38

# disk parameters (init_prim's first call, init.nz_pn_bbh_disk.c:425-441)
ADIAB = 0.01
GRSCALE = 0.01
Q_EXP = 1.58
RIN_DISK = 2.0 * (SEPARATION + M_TOT)
RPMAX_DISK = 5.0 * (SEPARATION + M_TOT)


def pnbbh_desc(n, r_in=0.75 * SEPARATION, r_out=13.0 * SEPARATION, r0=0.0, gam=5.0 / 3.0, cour=0.8, dt0=1.0e-5,
               t_final=1.0e4, precision=PREC_FP64, device=0):
    """GridDesc of the disk run on n = (N1, N2, N3) zones (init_base,
    init.nz_pn_bbh_disk.c:100-200), metric_dim 3."""
    n1, n2, n3 = (int(x) for x in n)
    length = [t_final, math.log((r_out - r0) / (r_in - r0)), 1.0, 2.0 * math.pi]
    dx = [dt0, length[1] / n1, length[2] / n2, length[3] / n3]
    startx = [0.0, math.log(r_in - r0) - NG * dx[1], 0.0 - NG * dx[2], 0.0 - NG * dx[3]]
    return make_desc((n1, n2, n3), gam, cour, dx, startx, length, recon=RECON_PPM_MC, flux=FLUX_HLLE, ct_para=1,
                     bc=BC_SPHERICAL_OUTFLOW3, metric_dim=3, use_ee=1, cooling=1, rescale_r=1, precision=precision,
                     device=device)


def pnbbh_coords(r0=0.0, **kw):
    """hg_dyn_metric with the grid's COORD_DIAGONAL3 parameters
    (diag3_factor = 1 - 2 th_cutout/pi - h_slope); further keywords (the
    spacetime and its parameters) go to dyn_metric()."""
    return dyn_metric(R0=r0, h_slope=H_SLOPE, diag3_exponent=DIAG3_EXPONENT, th_cutout=TH_CUTOUT, **kw)


def pnbbh_tables(desc, h_o_r=0.1, r0=0.0):
    """Per-zone floors and coordinates, FACE1 radii and the H/R cooling tables
    at the zones' own radii: the spacetime-independent output of the host
    builder (its static a = 0 Kerr-Schild geometry is not used)."""
    d2 = copy.copy(desc)
    d2.metric_dim = 2
    t = ks_mks_tables(d2, SPIN, R0=r0, h_slope=H_SLOPE, th_cutout=TH_CUTOUT, diag3_exponent=DIAG3_EXPONENT,
                      h_o_r=h_o_r)
    return dict(cell6=t["cell6"], rface=t["rface"], cool_omega=t["cool_omega"], cool_temp=t["cool_temp"])


# ---------------------------------------------------------------------------
# ranc() (ranc.c): 64 lanes S[n] <- S[n] * a[n] mod P[n] over primes just
# below 2^15.5, the next lane picked by the low 6 bits of the last state;
# seeding draws a[] and S[] from the C library's rand() after srand(seed).
_RANC_P = (46337, 46327, 46309, 46307, 46301, 46279, 46273, 46271, 46261, 46237, 46229, 46219, 46199, 46187, 46183,
           46181, 46171, 46153, 46147, 46141, 46133, 46103, 46099, 46093, 46091, 46073, 46061, 46051, 46049, 46027,
           46021, 45989, 45979, 45971, 45959, 45953, 45949, 45943, 45893, 45887, 45869, 45863, 45853, 45841, 45833,
           45827, 45823, 45821, 45817, 45779, 45767, 45763, 45757, 45751, 45737, 45707, 45697, 45691, 45677, 45673,
           45667, 45659, 45641, 45631)


class Ranc:
    """The reference's ranc(): Ranc(seed) is the call ranc(seed) (it seeds
    and returns one deviate, kept in .first); calling the object is ranc(0)."""

    def __init__(self, seed):
        libc = ctypes.CDLL(ctypes.util.find_library("c"))
        libc.rand.restype = ctypes.c_int
        libc.srand(ctypes.c_uint(seed))
        lo = 2 << 8
        self.a, self.s = [], []
        for p in _RANC_P:
            v = libc.rand() & 0x7FFF
            while v < lo or v > p - lo:
                v = libc.rand() & 0x7FFF
            self.a.append(v)
            w = libc.rand() & 0x7FFF
            while w < 1:
                w = libc.rand() & 0x7FFF
            self.s.append(w)
        self.n = 0
        self.first = self()

    def __call__(self):
        n = self.s[self.n] & 63
        self.n = n
        self.s[n] = (self.s[n] * self.a[n]) % _RANC_P[n]
        return float(self.s[n]) / float(_RANC_P[n])


# ---------------------------------------------------------------------------
# Boyer-Lindquist metric of mass M, spin a (bl_gcov_func / bl_gcon_func,
# metric.c:542-685), the components the disk needs, and trigvalues()
# (metric.c:29-41).
def _trig(th):
    sth, cth = math.sin(th), math.cos(th)
    if abs(sth) < SINGSMALL:
        sth = SINGSMALL if sth >= 0 else -SINGSMALL
    return cth, sth


def bl_metric(r, th, mass=M_TOT, spin=SPIN):
    """(gcov_tt, gcov_tp, gcov_pp, gcon_tt, gcon_tp, gcon_pp) at (r, th)."""
    cth, sth = _trig(th)
    t1 = mass * r
    t2 = r * r
    t3 = spin * spin
    t5 = cth * cth
    t7 = t2 + t3 * t5
    t8 = 1 / t7
    t14 = sth * sth
    t18 = 2.0 * mass * spin * r * t14 * t8
    t24 = t2 * t2
    gcov_tt = -1.0 + 2.0 * t1 * t8
    gcov_tp = -t18
    gcov_pp = t14 * t8 * (t24 + ((2.0 - t14) * t2 + (1.0 - t14) * t3) * t3 + 2.0 * t3 * t14 * t1)
    u1 = r * r
    u2 = u1 * u1
    u4 = cth * cth
    u7 = spin * spin
    u8 = u7 * u4
    u17 = 1 / (u1 + u8)
    u20 = 2.0 * mass * r
    u21 = -u1 + u20 - u7
    u22 = 1 / u21
    u28 = 2.0 * spin * mass * r * u17 * u22
    u33 = sth * sth
    gcon_tt = -(-u2 + ((-1.0 - u4) * u1 - u8) * u7 + 2.0 * (u4 - 1.0) * r * u7 * mass) * u17 * u22
    gcon_tp = u28
    gcon_pp = (-u1 - u8 + u20) * u22 * u17 / u33
    return gcov_tt, gcov_tp, gcov_pp, gcon_tt, gcon_tp, gcon_pp


def _radius_of_r(r, r0=0.0):
    """x[RR] of coord_of_r(r) on the COORD_DIAGONAL3 grid: x1 = log(r - R0),
    r = R0 + exp(x1) (xp_at_eq, coord.c:390-420); the equator th = pi/2."""
    return r0 + math.exp(math.log(r - r0))


def _sqrt(x):
    """C's sqrt: NaN for a negative argument (rho_func's radicands go negative
    near the axis; the NaN then fails h > 1 and the zone is outside the disk)."""
    return math.sqrt(x) if x >= 0. else math.nan


def _pow(x, y):
    """C's pow for the cases rho_func meets: NaN propagates, a negative base
    with a non-integer exponent gives NaN."""
    try:
        return math.pow(x, y)
    except ValueError:
        return math.nan


def _div(a, b):
    """C's division of doubles: a zero divisor gives +-inf or NaN."""
    try:
        return a / b
    except ZeroDivisionError:
        return math.nan if (a == 0. or a != a) else math.copysign(math.inf, a) * math.copysign(1., b)


class _Disk:
    """rho_func, get_rpmax, find_l_bracket, find_l_ang_in with the reference's
    shared state (init.nz_pn_bbh_disk.c:668-974)."""

    def __init__(self, gam, ranc, rin=RIN_DISK, rpmax=RPMAX_DISK, q=Q_EXP, adiab=ADIAB, grscale=GRSCALE,
                 mass=M_TOT, spin=SPIN, r0=0.0):
        self.gam, self.ranc, self.rin, self.rpmax, self.q = gam, ranc, rin, rpmax, q
        self.adiab, self.grscale, self.mass, self.spin, self.r0 = adiab, grscale, mass, spin, r0
        self.alpha = q / (q - 2.)
        self.exp_4 = self.alpha + 1.
        self.exp_2 = 1. / self.exp_4
        self.exp_3 = 1. / self.alpha
        self.geom_in = self.bl_at(rin)

    def bl_at(self, r):
        x = _radius_of_r(r, self.r0)
        return x, bl_metric(x, 0.5 * math.pi, self.mass, self.spin)

    def rho_func(self, xr, g, l_in):
        """(rho, uu, utcov, l_ang, utcon, upcon); rho = uu = -1 outside."""
        q, gam = self.q, self.gam
        gi = self.geom_in[1]
        sign_l = 1. if l_in >= 0. else -1.
        lambda_in = _sqrt(-gi[3] / gi[5])
        eta = abs(l_in) * _pow(lambda_in, (q - 2.))
        eta_2q = sign_l * _pow(eta, 2. / q)
        k_eta = _pow(eta, (-2. / (q - 2.)))
        f_l_in = _pow(abs(1. - k_eta * _pow(l_in, self.exp_4)), self.exp_2)
        utcov_in = _div(-1., _sqrt(-gi[3] + l_in * (2 * gi[4] - l_in * gi[5])))
        lam = _sqrt(-g[3] / g[5])
        omega = eta * _pow(lam, -q)
        l_ang = eta_2q * _pow(omega, self.exp_3)
        f_l = _pow(abs(1. - k_eta * _pow(l_ang, self.exp_4)), self.exp_2)
        utcov = _div(-1., _sqrt(-g[3] + l_ang * (2 * g[4] - l_ang * g[5])))
        utcon = _div(1., _sqrt(-(g[0] + omega * (2. * g[1] + omega * g[2]))))
        upcon = omega * utcon
        h = _div(utcov_in * f_l_in, utcov * f_l)
        if h > 1. and xr > self.rin:
            eps = (h - 1.) / gam
            rho = _pow((eps * (gam - 1.) / self.adiab), (1. / (gam - 1.)))
            uu = rho * eps * (1. + self.grscale * (self.ranc() - 0.5))
        else:
            rho = uu = -1.
        return rho, uu, utcov, l_ang, utcon, upcon

    def rho_at(self, r, l):
        x, g = self.bl_at(r)
        return self.rho_func(x, g, l)[0]

    def get_rpmax(self, l):
        r_lo = self.rin
        dr_frac = 1.e-3
        dr_big = 0.5
        dr = dr_big * dr_frac
        r = r_lo
        rho1 = self.rho_at(r, l)
        rho2 = self.rho_at(r + dr, l)
        drho_lo = (rho2 - rho1) / dr
        while True:
            dr_big *= 2
            r_hi = r_lo + dr_big
            r = r_hi
            dr = dr_big * dr_frac
            rho1 = self.rho_at(r - dr, l)
            rho2 = self.rho_at(r + dr, l)
            drho_hi = 0.5 * (rho2 - rho1) / dr
            done = drho_lo * drho_hi < 0.
            if r_hi > (self.mass * R_DISK_MAX):
                return -1.
            if done:
                break
        while True:
            dr_big = r_hi - r_lo
            r = 0.5 * (r_hi + r_lo)
            dr = dr_big * dr_frac
            rho1 = self.rho_at(r - dr, l)
            rho2 = self.rho_at(r + dr, l)
            drho = 0.5 * (rho2 - rho1) / dr
            if drho >= 0.:
                r_lo = r
            else:
                r_hi = r
            if drho == 0. or (dr_big / r) < 0.1 * L_ANG_PRECISION:
                break
        return r_lo

    def find_l_bracket(self):
        m, at = self.mass, self.spin / self.mass
        x = math.sqrt(self.rin / m)
        xsq = x * x
        l_lo = m * (xsq * (xsq - 2. * at) + at * at) / (x * (xsq - 2.) + at)
        x = math.sqrt(self.rpmax / m)
        xsq = x * x
        l_hi = m * (xsq * (xsq - 2. * at) + at * at) / (x * (xsq - 2.) + at)
        r_lo = self.get_rpmax(l_lo)
        r_hi = self.get_rpmax(l_hi)
        if r_lo < 0. and r_hi < 0.:
            raise RuntimeError("find_l_bracket: no bracket")
        if r_lo > 0. and r_lo < self.rpmax and r_hi > self.rpmax:
            return l_lo, l_hi
        if r_lo < 0.:
            r_lo, l_lo = r_hi, l_hi
        else:
            r_hi, l_hi = r_lo, l_lo
        if r_hi > self.rpmax:
            while True:
                l_lo -= 0.01 * l_lo
                r_lo = self.get_rpmax(l_lo)
                if r_lo < self.rpmax or abs(l_lo) > L_DISK_MAX * m or l_lo * l_hi < 0.:
                    break
            if r_lo > self.rpmax:
                raise RuntimeError("find_l_bracket: lower bound failed")
        else:
            while True:
                l_hi += 0.01 * l_hi
                r_hi = self.get_rpmax(l_hi)
                if r_hi > self.rpmax or abs(l_hi) > L_DISK_MAX * m or l_lo * l_hi < 0.:
                    break
            if r_hi < self.rpmax:
                raise RuntimeError("find_l_bracket: upper bound failed")
        return l_lo, l_hi

    def find_l_ang_in(self):
        l_lo, l_hi = self.find_l_bracket()
        rp_lo = self.get_rpmax(l_lo)
        rp_hi = self.get_rpmax(l_hi)
        while True:
            l = 0.5 * (l_lo + l_hi)
            r = self.get_rpmax(l)
            if r > self.rpmax:
                rp_hi, l_hi = r, l
            else:
                rp_lo, l_lo = r, l
            dr = abs((rp_hi - rp_lo) / self.rpmax)
            dl = abs(2. * (l_hi - l_lo) / (l_hi + l_lo))
            if min(dl, dr) < L_ANG_PRECISION:
                break
        l = 0.5 * (l_lo + l_hi)
        r = self.get_rpmax(l)
        if abs(r - self.rpmax) > 1.e-3 * abs(self.rpmax):
            raise RuntimeError("find_l_ang_in: pressure maximum at %g, not %g" % (r, self.rpmax))
        return l


def disk_fields(desc, tables, gam=5.0 / 3.0, seed=1):
    """init_data()'s zone loop (init.nz_pn_bbh_disk.c:216-240, 405-533) on the
    physical zones: rho, u, the BL 4-velocity (u^t, u^phi), the mask of zones
    inside the disk, and rho_max, u_max.  The random stream runs as the
    reference's does: ranc(seed), then the disk parameters' searches, then
    one deviate per physical zone inside the disk in (i, j, k) order."""
    n1, n2, n3 = desc.n1, desc.n2, desc.n3
    ranc = Ranc(seed)
    disk = _Disk(gam, ranc)
    l_in = disk.find_l_ang_in()
    x, g = disk.bl_at(disk.rpmax)
    disk.rho_func(x, g, l_in)            # rho_pmax (printed only): one more deviate
    c6 = np.asarray(tables["cell6"])
    rho = np.full((n1, n2), -1.0)
    eps_fac = np.zeros((n1, n2))
    ut = np.zeros((n1, n2))
    up = np.zeros((n1, n2))
    inside = np.zeros((n1, n2), bool)
    for i in range(n1):
        for j in range(n2):
            xr = float(c6[NG + i, NG + j, NG, 3]) + M_TOT
            th = float(c6[NG + i, NG + j, NG, 4])
            gb = bl_metric(xr, th)
            # rho_func without the deviate: the zone's draws are taken below in loop order
            save, disk.ranc = disk.ranc, (lambda: 0.5)
            r_, u_, _, _, utc, upc = disk.rho_func(xr, gb, l_in)
            disk.ranc = save
            if r_ > 0.:
                inside[i, j] = True
                rho[i, j] = r_
                eps_fac[i, j] = u_          # rho * eps (the factor at deviate 0.5 is exactly 1)
                ut[i, j], up[i, j] = utc, upc
    nin = int(inside.sum()) * n3
    dev = np.fromiter((ranc() for _ in range(nin)), float, nin)
    u = np.full((n1, n2, n3), -1.0)
    sel = np.broadcast_to(inside[:, :, None], (n1, n2, n3))
    u[sel] = (np.broadcast_to(eps_fac[:, :, None], (n1, n2, n3))[sel] * (1. + GRSCALE * (dev - 0.5)))
    rho3 = np.broadcast_to(rho[:, :, None], (n1, n2, n3))
    rho_max = max(0.0, float(rho.max()))
    u_max = max(0.0, float(np.where(sel, u, 0.0).max()))
    return dict(rho=rho3, u=u, ut=ut, up=up, inside=inside, rho_max=rho_max, u_max=u_max, l_ang_in=l_in)


def _bsq(pr, geo):
    """bsq_calc (phys.c:190-296) of one zone's primitives pr[8] with the
    struct of_geom geo[42], in the reference's operation order."""
    gc = geo[G_GCOV:G_GCOV + 16]
    u1, u2, u3 = pr[2], pr[3], pr[4]
    qsq = (gc[5] * u1 * u1 + gc[10] * u2 * u2 + gc[15] * u3 * u3
           + 2 * (gc[6] * u1 * u2 + gc[7] * u1 * u3 + gc[11] * u2 * u3))
    if qsq < 0.:
        if abs(qsq) > 1.e-10:
            raise RuntimeError("gamma_calc failed in the field normalisation")
        qsq = 1.e-10
    gamma = math.sqrt(1. + qsq)
    ucon = [gamma * geo[G_NCON], 0., 0., 0.]
    for a in range(3):
        ucon[a + 1] = pr[2 + a] - ucon[0] * geo[G_BETA + a]

    def lower(v):
        return [gc[4 * a] * v[0] + gc[4 * a + 1] * v[1] + gc[4 * a + 2] * v[2] + gc[4 * a + 3] * v[3]
                for a in range(4)]

    ucov = lower(ucon)
    inv_ut = 1. / ucon[0]
    b0 = pr[5] * ucov[1] + pr[6] * ucov[2] + pr[7] * ucov[3]
    bcon = [b0, (pr[5] + b0 * ucon[1]) * inv_ut, (pr[6] + b0 * ucon[2]) * inv_ut, (pr[7] + b0 * ucon[3]) * inv_ut]
    bcov = lower(bcon)
    return bcon[0] * bcov[0] + bcon[1] * bcov[1] + bcon[2] * bcov[2] + bcon[3] * bcov[3]


def _omega_circular(r, mass=M_TOT, spin=SPIN):
    """omega_circular_equatorial (phys.c:861-905) with r_isco = 0 (the
    setup's, init.nz_pn_bbh_disk.c:326)."""
    return math.sqrt(mass) / (math.pow(r, 1.5) + spin)


def _target_temperature(r, h_o_r, spin=SPIN):
    """target_temperature (phys.c:805-848) outside r_isco = 0."""
    rm1 = 1. / r
    x = math.sqrt(r)
    xm3 = 1. / (x * x * x)
    term1 = spin * spin * rm1
    c_f = 1. - 3 * rm1 + 2 * spin * xm3
    f_f = 1. - 2 * spin * xm3 + term1 * rm1
    g_f = 1. - 2 * rm1 + spin * xm3
    ut_sq = g_f * g_f / c_f
    uphi_sq = f_f * f_f * r / c_f
    r_z = uphi_sq * rm1 - term1 * (ut_sq - 1.)
    return 0.5 * math.pi * r_z * h_o_r * h_o_r * rm1


def pn_cooling_tables(tables, h_o_r=0.1):
    """Cooling tables of a run in a post-Newtonian (harmonic-coordinate)
    metric: the reference takes Omega and T at the Boyer-Lindquist radius
    r + M there (USE_ISOTROPIC_COORDS, phys.c:829-831, 888-891), along the
    row (i, N2S, N3S) it tabulates (phys.c:683-704)."""
    c6 = np.asarray(tables["cell6"])
    om = np.array([_omega_circular(float(r) + M_TOT) for r in c6[:, NG, NG, 3]])
    tt = np.array([_target_temperature(float(r) + M_TOT, h_o_r) for r in c6[:, NG, NG, 3]])
    return om, tt


def set_disk(target, desc, tables, metric, beta=10.0, seed=1, t0=0.0, return_prims=True, plane_batch=16):
    """Initial data of the circumbinary disk on `target` (init_data,
    init.nz_pn_bbh_disk.c:216-300) for the grid metric `metric` (an
    hg_dyn_metric) at time t0: the disk fields, their 4-velocity turned into
    primitives with the grid's gcon at the zone centres, fixup(p); bounds(p,0),
    the dipole loop normalised to plasma beta `beta`, fixup(p); bounds(p,0).
    `target` is anything with upload(p), fixup_bounds() and download() -- an
    Engine, whose floors and boundary kernels are the ones the step uses.
    Returns (primitives in the reference layout or None, disk fields)."""
    from . import dyn_geometry_block
    n1, n2, n3 = desc.n1, desc.n2, desc.n3
    shp = ref_shape((n1, n2, n3))
    h = disk_fields(desc, tables, desc.gam, seed)
    p = np.zeros(shp + (8,))
    inside = h["inside"]
    # ucon = (u^t, 0, 0, u^phi) in (r, th, phi) is unchanged by the diagonal
    # COORD_DIAGONAL3 map (transform_rank1con2); ucon2pr with the grid metric
    for i0 in range(0, n1, plane_batch):
        ni = min(plane_batch, n1 - i0)
        if not inside[i0:i0 + ni].any():
            continue
        geo = dyn_geometry_block(desc, metric, CENT, t0, NG + i0, ni)[:, NG:NG + n2, NG:NG + n3]
        gcon = geo[..., G_GCON:G_GCON + 4]
        m = np.broadcast_to(inside[i0:i0 + ni, :, None], (ni, n2, n3))
        ut = np.broadcast_to(h["ut"][i0:i0 + ni, :, None], (ni, n2, n3))
        up = np.broadcast_to(h["up"][i0:i0 + ni, :, None], (ni, n2, n3))
        f = ut / gcon[..., 0]
        blk = p[NG + i0:NG + i0 + ni, NG:NG + n2, NG:NG + n3]
        blk[..., 0] = np.where(m, h["rho"][i0:i0 + ni], 0.0)
        blk[..., 1] = np.where(m, h["u"][i0:i0 + ni], 0.0)
        blk[..., 2] = np.where(m, 0.0 - gcon[..., 1] * f, 0.0)
        blk[..., 3] = np.where(m, 0.0 - gcon[..., 2] * f, 0.0)
        blk[..., 4] = np.where(m, up - gcon[..., 3] * f, 0.0)
    target.upload(p)
    target.fixup_bounds()
    p = target.download()

    # set_mag_field: A_phi at the corners (i, j) = N1S..N1E+1, N2S..N2E+1 of the
    # k = N3S slice, B on the k = 0 layer with its sqrt(-g), the integrals in
    # the reference's (i, j) order
    rk = p[:, :, NG, 0]
    i0, i1, j0, j1 = NG, NG + n1 + 1, NG, NG + n2 + 1
    rho_avg = 0.25 * (rk[i0:i1, j0:j1] + rk[i0 - 1:i1 - 1, j0:j1] + rk[i0:i1, j0 - 1:j1 - 1] +
                      rk[i0 - 1:i1 - 1, j0 - 1:j1 - 1])
    rho_cut = 0.25 * h["rho_max"]
    A = np.where(rho_avg > rho_cut, rho_avg - rho_cut, 0.0)
    geo0 = np.concatenate([dyn_geometry_block(desc, metric, CENT, t0, NG + i0, min(plane_batch, n1 - i0))[:, NG:NG + n2, 0]
                           for i0 in range(0, n1, plane_batch)])
    gdet = geo0[..., G_G]
    b1 = -(A[:-1, :-1] - A[:-1, 1:] + A[1:, :-1] - A[1:, 1:]) / (2. * desc.dx[2] * gdet)
    b2 = (A[:-1, :-1] + A[:-1, 1:] - A[1:, :-1] - A[1:, 1:]) / (2. * desc.dx[1] * gdet)
    bsq_int = u_int = 0.
    for i in range(n1):
        for j in range(n2):
            pr = p[NG + i, NG + j, 0].copy()
            pr[5], pr[6], pr[7] = b1[i, j], b2[i, j], 0.
            g = float(gdet[i, j])
            bsq_int += g * _bsq(pr, geo0[i, j])
            u_int += g * float(pr[1])
    beta_act = (desc.gam - 1.) * u_int / (0.5 * bsq_int)
    norm = math.sqrt(beta_act / beta)
    p[NG:NG + n1, NG:NG + n2, 0, 5] = b1 * norm
    p[NG:NG + n1, NG:NG + n2, 0, 6] = b2 * norm
    p[NG:NG + n1, NG:NG + n2, 0, 7] = 0.
    p[:, :, :, 5:8] = p[:, :, 0:1, 5:8]
    target.upload(p)
    target.fixup_bounds()
    return (target.download() if return_prims else None), h
