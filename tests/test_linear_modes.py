"""Exact RMHD linear eigenmodes (setups.rmhd_modes / eigenmode) and the 3D
linear-wave problem built on them (setups.linear_wave_3d).

Pins: the reference's closed-form slow, Alfven and fast modes (eigs(),
init.linearwave.c:166-240, restated below for B = (Bx, 0, 0), Gamma 4/3,
rho 1, u 1/(Gamma - 1), k = 2 pi (1, 1, 0)) are reproduced by the numerical
eigensolver, eigenvalue and eigenvector; and the speeds of the oblique
configuration (B = (1, 1.5, 0) along the grid diagonal) meet the analytic
RMHD speeds of a static medium (Alfven B_n / sqrt(rho h + B^2), fast
perpendicular sqrt(vA^2 + cs^2 (1 - vA^2)), sound and Alfven for B along
the wave).  On the GPU the engine runs the oblique fast wave bit for bit like
the C oracle, and its errors fall at second order with MC reconstruction."""
import math

import numpy as np
import pytest

import coolharm3d_b200 as hg
import harmtest as ht
from coolharm3d_b200 import convergence, setups

GAM = 4.0 / 3.0


def reference_eigs(Bx, branch):
    """eigs() of init.linearwave.c (SLOW / ALFVEN / FAST branches): the
    frequency w and the primitive perturbation dp for k = 2 pi (1, 1, 0)."""
    dp = np.zeros(8)
    Bx2 = Bx * Bx
    if branch == "alfven":
        dp[4] = -1.0 / math.sqrt(5.0 + Bx2)
        dp[7] = 1.0
        return 2.0 * math.pi * Bx / math.sqrt(5.0 + Bx2), dp
    aux1 = 400.0 + 80.0 * Bx2 + 169.0 * Bx2 * Bx2
    r1 = 2.0 * math.pi * math.sqrt((20.0 + 17.0 * Bx2 - math.sqrt(aux1)) / (75.0 + 15.0 * Bx2))
    r2 = 2.0 * math.pi * math.sqrt((20.0 + 17.0 * Bx2 + math.sqrt(aux1)) / (75.0 + 15.0 * Bx2))
    first = (r2 > r1) if branch == "slow" else (r1 > r2)
    s = 1.0 if first else -1.0
    dp[0] = (-20.0 + 13 * Bx2 + s * math.sqrt(aux1)) / 20.0
    dp[1] = (-20.0 + 13 * Bx2 + s * math.sqrt(aux1)) / 5.0
    dp[2] = math.sqrt((20.0 + 17.0 * Bx2 - s * math.sqrt(aux1)) / (75.0 + 15.0 * Bx2)) * \
        (13.0 * Bx2 + s * math.sqrt(aux1)) / 20.0
    dp[3] = -math.sqrt((20.0 + 17.0 * Bx2 - s * math.sqrt(aux1)) / (75.0 + 15.0 * Bx2))
    dp[5] = -Bx
    dp[6] = Bx
    return (r1 if first else r2), dp


@pytest.mark.parametrize("branch", ["slow", "alfven", "fast"])
@pytest.mark.parametrize("Bx", [0.5, 1.0, 2.0])
def test_eigensolver_reproduces_reference_closed_forms(branch, Bx):
    w_ref, dp_ref = reference_eigs(Bx, branch)
    dp, lam = setups.eigenmode(branch, 1.0, 1.0, GAM, (Bx, 0.0, 0.0), (1, 1, 0))
    assert abs(2.0 * math.pi * math.sqrt(2.0) * lam - w_ref) <= 1e-13 * w_ref
    dp_ref = dp_ref / dp_ref[np.argmax(np.abs(dp_ref))]
    np.testing.assert_allclose(dp, dp_ref, rtol=1e-12, atol=1e-13)


def test_oblique_speeds_meet_analytic_rmhd_speeds():
    B = np.array([1.0, 1.5, 0.0])
    nhat = np.ones(3) / math.sqrt(3.0)
    rho_h = 1.0 + 3.0 + 1.0          # rho + u + p
    lam, _ = setups.rmhd_modes(1.0, 1.0, GAM, B, (1, 1, 1))
    assert abs(lam[5] - B @ nhat / math.sqrt(rho_h + B @ B)) <= 1e-14
    assert lam[3] == pytest.approx(0.0, abs=1e-15)
    np.testing.assert_allclose(lam[:3], -lam[4:][::-1], rtol=1e-13)
    assert lam[4] < lam[5] < lam[6] < 1.0
    cs2 = GAM * 1.0 / rho_h
    Bp = np.array([0.0, 1.5, 0.0])   # field normal to the wave
    lam, _ = setups.rmhd_modes(1.0, 1.0, GAM, Bp, (1, 0, 0))
    va2 = Bp @ Bp / (rho_h + Bp @ Bp)
    assert abs(lam[6] - math.sqrt(va2 + cs2 * (1.0 - va2))) <= 1e-14
    lam, _ = setups.rmhd_modes(1.0, 1.0, GAM, (1.5, 0.0, 0.0), (1, 0, 0))   # field along the wave
    assert {round(lam[4], 13), round(lam[6], 13)} == {round(math.sqrt(cs2), 13), round(math.sqrt(va2), 13)}


def test_oblique_mode_structure():
    nhat = np.ones(3) / math.sqrt(3.0)
    for mode in ("fast", "alfven", "slow"):
        dp, lam = setups.eigenmode(mode, 1.0, 1.0, GAM, (1.0, 1.5, 0.0), (1, 1, 1))
        assert dp.max() == 1.0
        assert abs(dp[5:] @ nhat) <= 1e-14, mode          # no normal field perturbation
    dp, _ = setups.eigenmode("alfven", 1.0, 1.0, GAM, (1.0, 1.5, 0.0), (1, 1, 1))
    assert dp[0] == 0.0 and dp[1] == 0.0
    assert abs(dp[2:5] @ nhat) <= 1e-14                   # transverse velocity
    assert abs(dp[2:5] @ np.array([1.0, 1.5, 0.0])) <= 1e-14
    with pytest.raises(ValueError):
        setups.eigenmode("alfven", 1.0, 1.0, GAM, (1.0, 1.0, 1.0), (1, 1, 1))   # degenerate with the fast mode


def test_linear_wave_3d_initial_state():
    prob = setups.linear_wave_3d((8, 8, 8))
    dp, lam = setups.eigenmode("fast", 1.0, 1.0, GAM, (1.0, 1.5, 0.0), (1, 1, 1))
    assert prob.t_final == pytest.approx(1.0 / (math.sqrt(3.0) * lam), rel=1e-15)
    assert prob.desc.grid_length[0] == prob.t_final
    p = prob.p_init
    phys = p[3:11, 3:11, 3:11]
    # whole wavelengths in the box: the perturbation averages to zero
    np.testing.assert_allclose(phys.reshape(-1, 8).mean(0), [1.0, 3.0, 0, 0, 0, 1.0, 1.5, 0.0], atol=1e-14)
    x = (np.array([3, 5, 7]) - 3 + 0.5) / 8.0
    expect = np.array([1.0, 3.0, 0, 0, 0, 1.0, 1.5, 0.0]) + 1e-6 * dp * math.cos(2.0 * math.pi * x.sum())
    np.testing.assert_allclose(p[3, 5, 7], expect, rtol=1e-15, atol=1e-21)
    assert not p[:3].any() and not p[11:].any()            # ghosts come from bounds()
    with pytest.raises(ValueError):
        setups.linear_wave_3d((8, 8, 1))                   # k3 != 0 on a one-zone x3


def test_wave_vars():
    assert convergence.wave_vars("alfven") == ("U1", "U2", "U3", "B1", "B2", "B3")
    assert convergence.wave_vars("alfven", dims=2) == ("U3", "B3")
    assert convergence.wave_vars("fast") == convergence.VARS


def _oracle(prob):
    d = prob.desc
    sw = dict(recon=d.recon_type, flux=d.flux_type, ct_para=d.use_flux_ct_para, bc=d.bc_type, metric_dim=0,
              ee=d.use_entropy_eq, cooling=0, rescale=0)
    geomd = dict(gam=d.gam, cour=d.cour, grid_length=np.array(d.grid_length[:]), startx=np.array(d.startx[:]),
                 dx=np.array(d.dx[:]), geom=prob.geom, conn=np.zeros(1), cell6=prob.cell6, rface=None)
    return ht.Oracle(prob.n, sw, geomd, lib=ht.CR_ORACLE)


@pytest.mark.gpu
@pytest.mark.parametrize("mode,n", [("fast", (12, 10, 8)), ("alfven", (8, 8, 8))])
def test_engine_matches_oracle_on_oblique_wave(mode, n):
    prob = setups.linear_wave_3d(n, mode, kvec=(1, 1, 1))
    o = _oracle(prob)
    o.upload(prob.p_init)
    o.fixup_bounds()
    o.set_state(o.download(), 0.0, prob.desc.dx[0])
    e = hg.Engine(prob.desc)
    setups.start(e, prob)
    o.step(5)
    t, dt = e.step(5)
    ref = o.state()
    np.testing.assert_array_equal(e.download(), ref["p"])
    assert (t, dt) == (ref["t"], ref["dt"])
    assert e.fail_counts().tolist() == ref["nfailtot"].tolist()
    e.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["fast", "alfven"])
def test_oblique_modes_converge_at_second_order_with_mc(mode):
    out = convergence.study(sizes=(16, 32, 64), dims=3, mode=mode, recon=hg.RECON_MC)
    print(out["order"])
    for o in out["order"]:
        assert min(o.values()) > 1.7, o


@pytest.mark.gpu
def test_oblique_fast_mode_ppm_and_mixed():
    """PPM_MC (the configuration's scheme) reduces the error from 16^3 to
    32^3, and the mixed form stays within L1 1e-6 of the exact mode."""
    fp = convergence.study(sizes=(16, 32), dims=3, mode="fast")
    mx = convergence.study(sizes=(32,), dims=3, mode="fast", precision=hg.PREC_MIXED)
    print(fp["order"], mx["errors"])
    assert min(fp["order"][0].values()) > 1.0
    assert max(mx["errors"][0].values()) < 1e-6
