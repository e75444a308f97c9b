"""Pins the oracle's advective operator (advective_swm_operator, covariant Ch
branch: up4 mass flux on the interpolating ECS_xy halo, up4 vector advection on
the bicubic ECS vector halo, Christoffel terms, edge sync of the tendencies) by
known-answer properties; the linear operator these reduce to is pinned in
tests/test_oracle.py."""
import numpy as np
import pytest

from oracle.oracle import EARTH_GRAV, EARTH_RADIUS, Oracle

H0 = 29400 / EARTH_GRAV


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def smooth_state(o, seed, amp_u=10.0):
    """A smooth wind (solid rotation about a random axis) and a smooth h perturbation."""
    rng = np.random.default_rng(seed)
    axis = rng.standard_normal(3)
    axis /= np.linalg.norm(axis)
    _, u, v = o.ts2(u0=amp_u, h_mean=0.0, axis=axis, linear_mode=True)
    eta = o.zeros()[0]
    for _ in range(3):
        eta += o.gaussian(lam0=rng.uniform(0, 2 * np.pi), phi0=np.arcsin(rng.uniform(-1, 1)),
                          d0=rng.uniform(0.2, 0.5), amp=rng.uniform(-5, 5))[0]
    return eta, u, v


@pytest.fixture(scope="module")
def pair(oracle_built):
    return Oracle(20, h_mean=H0, operator="advective"), Oracle(20, h_mean=H0)


def test_rest_state_gives_gradient_wind_only(pair):
    nl, lin = pair
    eta, u, v = smooth_state(nl, 1)
    h = H0 + eta
    z = np.zeros_like(u), np.zeros_like(v)
    dh, du, dv = nl.apply(h, *z)
    dhl, dul, dvl = lin.apply(h, *z)
    assert np.abs(dh).max() == 0.0
    assert rel(du, dul) < 1e-13 and rel(dv, dvl) < 1e-13


def test_constant_depth_flux_matches_linear_divergence(pair):
    nl, lin = pair
    _, u, v = smooth_state(nl, 2)
    h = np.full(nl.zeros()[0].shape, H0)
    dh, _, _ = nl.apply(h, u, v)
    dhl, _, _ = lin.apply(h, u, v)
    assert rel(dh, dhl) < 1e-12


def test_linearisation_about_rest_is_the_linear_operator(pair):
    nl, lin = pair
    eta, u, v = smooth_state(nl, 3)
    base = nl.apply(np.full(eta.shape, H0), np.zeros_like(u), np.zeros_like(v))
    ref = lin.apply(eta, u, v)
    errs = []
    for eps in (1e-3, 5e-4):
        out = nl.apply(H0 + eps * eta, eps * u, eps * v)
        errs.append(max(rel((o - b) / eps, r) for o, b, r in zip(out, base, ref)))
    assert errs[0] < 1e-2
    assert 1.6 < errs[0] / errs[1] < 2.4      # first-order remainder: O(eps)


def test_mass_conserved(pair):
    nl, _ = pair
    eta, u, v = smooth_state(nl, 4, amp_u=30.0)
    dh, _, _ = nl.apply(H0 + eta, u, v)
    assert abs(nl.dot(0, dh)) < 1e-12 * nl.dot(0, np.abs(dh))
    h1, u1, v1 = nl.rk4(H0 + eta, u, v, 1200.0, 4)
    m0, _ = nl.integrals(H0 + eta, u, v)
    m1, _ = nl.integrals(h1, u1, v1)
    assert abs(m1 - m0) < 1e-13 * abs(m0)


def test_williamson2_steady_state_converges():
    """Williamson test 2 (tilted axis) is a steady state of the nonlinear equations:
    the error in h after 6 h falls at about third order."""
    axis = (np.sin(0.6), 0.0, np.cos(0.6))
    u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
    errs = []
    for N in (16, 32):
        o = Oracle(N, h_mean=H0, axis=axis, operator="advective")
        h, u, v = o.ts2(u0=u0, h_mean=H0, axis=axis)
        dt = 900.0 * 32 / N
        h1, _, _ = o.rk4(h, u, v, dt, int(round(6 * 3600.0 / dt)))
        errs.append(np.abs(h1 - h).max() / np.abs(h).max())
    assert errs[1] < 2e-4
    assert np.log2(errs[0] / errs[1]) > 2.3, errs


@pytest.mark.parametrize("order", [21, 63])
def test_advective_sbp_orders_conserve_mass_and_match_at_rest(order):
    """The advective operator with the 2-1 / 6-3 Ch operators: at rest its tendency is
    the linear operator's gradient wind of the same order (the advection and the
    Christoffel terms vanish), and RK4 conserves mass to round-off."""
    from oracle.oracle import Oracle
    N = 16
    o = Oracle(N, h_mean=1000.0, operator="advective", sbp_order=order)
    h = 1000.0 + o.gaussian(lam0=1.0, phi0=0.3, d0=0.4, amp=20.0)[0]
    _, u, v = o.zeros()
    dh, du, dv = o.apply(h, u, v)
    lin = Oracle(N, h_mean=1000.0, sbp_order=order)
    _, lu, lv = lin.apply(h - 1000.0, u, v)
    assert np.abs(du - lu).max() < 1e-12 * np.abs(lu).max() and np.abs(dv - lv).max() < 1e-12 * np.abs(lv).max()
    assert np.abs(dh).max() == 0.0
    m0 = o.integrals(h, u, v)[0]
    hs, us, vs = o.rk4(h, u, v, 600.0, 6)
    assert abs(o.integrals(hs, us, vs)[0] - m0) < 1e-13 * abs(m0)


def test_orography_enters_the_gradient_only():
    """operator_adv_swm_mod.f90:78: the gradient acts on h + h_surf, the mass flux on h.
    So with orography the wind tendency equals the one of the flat operator applied to
    h + h_surf, and the height tendency equals the flat operator's at h."""
    from ch_swe_b200.testcases import williamson5
    from oracle.oracle import Oracle
    N = 16
    h, u, v, hs = williamson5(N)
    o = Oracle(N, h_mean=5960.0, operator="advective")
    o.set_orography(hs)
    dh, du, dv = o.apply(h, u, v)
    o.set_orography(None)
    _, du_t, dv_t = o.apply(h + hs, u, v)
    dh_f, _, _ = o.apply(h, u, v)
    assert np.array_equal(dh, dh_f)
    for a, b in ((du, du_t), (dv, dv_t)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
