"""Pins the CPU oracle (oracle/swe_oracle.c) by known-answer properties of the
reference's discretisation (no Fortran toolchain or golden vectors exist for
this path, so these properties, not a binary, pin the restatement).
"""
import numpy as np
import pytest

from oracle.oracle import EARTH_GRAV, EARTH_RADIUS, Oracle


@pytest.fixture(scope="module", params=[42, 21, 63], ids=["sbp42", "sbp21", "sbp63"])
def o24(oracle_built, request):
    """C24 oracle with the SBP 4-2, 2-1 and 6-3 Ch operators."""
    return Oracle(24, sbp_order=request.param)


def smooth_h(o, seed, k=5):
    rng = np.random.default_rng(seed)
    h = o.zeros()[0]
    for _ in range(k):
        h += o.gaussian(lam0=rng.uniform(0, 2 * np.pi), phi0=np.arcsin(rng.uniform(-1, 1)),
                        d0=rng.uniform(0.2, 0.5), amp=rng.uniform(-1, 1))[0]
    return h


def test_gradient_of_constant_vanishes(o24):
    gx, gy = o24.grad(np.full(o24.zeros()[0].shape, 3.7))
    assert np.abs(gx).max() < 1e-18 and np.abs(gy).max() < 1e-18


def test_co2contra_symmetric_in_sbp_norm(o24):
    rng = np.random.default_rng(1)
    _, u, v = o24.zeros()
    a1, a2, b1, b2 = (rng.standard_normal(x.shape) for x in (u, v, u, v))
    ta1, ta2 = o24.co2contra(a1, a2)
    tb1, tb2 = o24.co2contra(b1, b2)
    lhs = o24.dot(1, a1, tb1) + o24.dot(2, a2, tb2)
    rhs = o24.dot(1, ta1, b1) + o24.dot(2, ta2, b2)
    assert abs(lhs - rhs) < 1e-13 * abs(lhs)


def test_sbp_adjointness_grad_div(o24):
    """<grad h, u^c>_u + <h, div u^c>_h = 0 for h continuous across panel edges."""
    rng = np.random.default_rng(2)
    h = smooth_h(o24, 3)
    _, u, v = o24.zeros()
    ut, vt = o24.co2contra(rng.standard_normal(u.shape), rng.standard_normal(v.shape))
    gx, gy = o24.grad(h)
    a = o24.dot(1, gx, ut) + o24.dot(2, gy, vt)
    b = o24.dot(0, h, o24.div(ut, vt))
    assert abs(a + b) < 1e-12 * abs(a)


def test_coriolis_energy_neutral(o24):
    rng = np.random.default_rng(4)
    _, u, v = o24.zeros()
    ut, vt = o24.co2contra(rng.standard_normal(u.shape), rng.standard_normal(v.shape))
    cu, cv = o24.coriolis(ut, vt)
    s = o24.dot(1, np.abs(cu), np.abs(ut)) + o24.dot(2, np.abs(cv), np.abs(vt))
    assert abs(o24.dot(1, cu, ut) + o24.dot(2, cv, vt)) < 1e-13 * s


def test_semidiscrete_energy_and_mass_conserved(o24):
    rng = np.random.default_rng(5)
    h = smooth_h(o24, 6)
    _, u, v = o24.zeros()
    u, v = rng.standard_normal(u.shape), rng.standard_normal(v.shape)
    dh, du, dv = o24.apply(h, u, v)
    ut, vt = o24.co2contra(u, v)
    terms = [o24.h_mean * o24.dot(1, du, ut), o24.h_mean * o24.dot(2, dv, vt), o24.grav * o24.dot(0, h, dh)]
    assert abs(sum(terms)) < 1e-10 * sum(abs(t) for t in terms)
    assert abs(o24.dot(0, dh)) < 1e-12 * o24.dot(0, np.abs(dh))


def test_mass_conserved_over_rk4(o24):
    h, u, v = o24.gaussian(lam0=1.0, phi0=0.3, d0=0.2)
    m0, _ = o24.integrals(h, u, v)
    h1, u1, v1 = o24.rk4(h, u, v, 900.0, 8)
    m1, _ = o24.integrals(h1, u1, v1)
    assert abs(m1 - m0) < 1e-13 * abs(m0)


def test_linear_williamson2_steady_state_converges(oracle_built):
    """Linear TS2 is an exact steady state; the error after 1/4 day falls at ~3rd order."""
    errs = []
    axis = (np.sin(0.7), 0.0, np.cos(0.7))
    for N in (16, 32):
        o = Oracle(N, h_mean=29400 / EARTH_GRAV, axis=axis)
        u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
        h, u, v = o.ts2(u0=u0, h_mean=29400 / EARTH_GRAV, axis=axis, linear_mode=True)
        dt = 900.0 * 32 / N                      # CFL ~ 0.5 for c = sqrt(gH) ~ 171 m/s
        nsteps = int(round(6 * 3600.0 / dt))
        h1, _, _ = o.rk4(h, u, v, dt, nsteps)
        errs.append(np.abs(h1 - h).max() / np.abs(h).max())
    order = np.log2(errs[0] / errs[1])
    assert order > 2.0, (errs, order)


def test_linear_williamson2_steady_state_converges_sbp21(oracle_built):
    """SBP 2-1 (second order inside, first at the panel edges): the TS2 error after
    1/4 day falls at better than first order."""
    errs = []
    axis = (np.sin(0.7), 0.0, np.cos(0.7))
    for N in (16, 32):
        o = Oracle(N, h_mean=29400 / EARTH_GRAV, axis=axis, sbp_order=21)
        u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
        h, u, v = o.ts2(u0=u0, h_mean=29400 / EARTH_GRAV, axis=axis, linear_mode=True)
        dt = 900.0 * 32 / N
        nsteps = int(round(6 * 3600.0 / dt))
        h1, _, _ = o.rk4(h, u, v, dt, nsteps)
        errs.append(np.abs(h1 - h).max() / np.abs(h).max())
    order = np.log2(errs[0] / errs[1])
    assert order > 1.0, (errs, order)


def test_linear_williamson2_steady_state_converges_sbp63(oracle_built):
    """SBP 6-3 (sixth order inside, third at the panel edges): the TS2 error after
    1/4 day falls at better than third order and below the 4-2 error at C32."""
    errs = []
    axis = (np.sin(0.7), 0.0, np.cos(0.7))
    for N in (16, 32):
        o = Oracle(N, h_mean=29400 / EARTH_GRAV, axis=axis, sbp_order=63)
        u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
        h, u, v = o.ts2(u0=u0, h_mean=29400 / EARTH_GRAV, axis=axis, linear_mode=True)
        dt = 900.0 * 32 / N
        nsteps = int(round(6 * 3600.0 / dt))
        h1, _, _ = o.rk4(h, u, v, dt, nsteps)
        errs.append(np.abs(h1 - h).max() / np.abs(h).max())
    order = np.log2(errs[0] / errs[1])
    assert order > 3.0, (errs, order)


@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_sbp63_polynomial_exactness(oracle_built, deg):
    """The 6-3 differences are exact for polynomials of degree <= 3, the
    interpolations for degree <= 2 (third-order closures); interior rows exact to
    degree 5."""
    from oracle.oracle import sbp1d
    n = 30
    xn = np.linspace(0.0, 1.0, n + 1)
    xc = 0.5 * (xn[:-1] + xn[1:])
    hx = xn[1] - xn[0]
    f = lambda x: x ** deg
    df = lambda x: deg * x ** (deg - 1) if deg else 0 * x
    assert np.allclose(sbp1d(0, n, f(xn), order=63) / hx, df(xc), atol=1e-11)
    assert np.allclose(sbp1d(1, n, f(xc), order=63) / hx, df(xn), atol=1e-11)
    if deg <= 2:
        assert np.allclose(sbp1d(2, n, f(xn), order=63), f(xc), atol=1e-12)
        assert np.allclose(sbp1d(3, n, f(xc), order=63), f(xn), atol=1e-12)
    g = lambda x: x ** 5
    inner = slice(8, n - 8)
    assert np.allclose(sbp1d(0, n, g(xn), order=63)[inner] / hx, 5 * xc[inner] ** 4, atol=1e-9)
    assert np.allclose(sbp1d(3, n, g(xc), order=63)[inner], g(xn)[inner], atol=1e-12)


@pytest.mark.parametrize("deg", [0, 1])
def test_sbp21_polynomial_exactness(oracle_built, deg):
    """The 2-1 differences are exact for polynomials of degree <= 1 and the
    interpolations for degree 0 everywhere and degree 1 away from the boundary rows."""
    from oracle.oracle import sbp1d
    n = 20
    xn = np.linspace(0.0, 1.0, n + 1)
    xc = 0.5 * (xn[:-1] + xn[1:])
    hx = xn[1] - xn[0]
    f = lambda x: x ** deg
    df = lambda x: deg * x ** (deg - 1) if deg else 0 * x
    assert np.allclose(sbp1d(0, n, f(xn), order=21) / hx, df(xc), atol=1e-12)
    assert np.allclose(sbp1d(1, n, f(xc), order=21) / hx, df(xn), atol=1e-12)
    assert np.allclose(sbp1d(2, n, f(xn), order=21), f(xc), atol=1e-12)
    assert np.allclose(sbp1d(3, n, f(xc), order=21)[1:-1], f(xn)[1:-1], atol=1e-12)


@pytest.mark.parametrize("deg", [0, 1, 2])
def test_sbp42_polynomial_exactness(oracle_built, deg):
    """SBP 4-2 including the closure rows: differences exact up to degree 2; the
    interpolations up to degree 1 (their free closure parameters c13, c14 minimise
    the degree-2 error instead, sbp_interp_i2c_42_mod.f90:12-19)."""
    from oracle.oracle import sbp1d
    n = 20
    xn = np.arange(n + 1, dtype=float)          # nodes 0..n
    xc = np.arange(n, dtype=float) + 0.5         # centres
    f = lambda x: (0.3 + 1.7 * x - 0.05 * x ** 2) if deg == 2 else (0.3 + 1.7 * x if deg == 1 else 0.3 + 0 * x)
    df = lambda x: (1.7 - 0.1 * x) if deg == 2 else (1.7 + 0 * x if deg == 1 else 0 * x)
    if deg <= 1:
        assert np.allclose(sbp1d(2, n, f(xn)), f(xc), atol=1e-12)
        assert np.allclose(sbp1d(3, n, f(xc)), f(xn), atol=1e-12)
    assert np.allclose(sbp1d(0, n, f(xn)), df(xc), atol=1e-12)
    assert np.allclose(sbp1d(1, n, f(xc)), df(xn), atol=1e-12)


def test_sbp42_interior_cubic_exactness(oracle_built):
    from oracle.oracle import sbp1d
    n = 24
    xn = np.arange(n + 1, dtype=float)
    xc = np.arange(n, dtype=float) + 0.5
    f = lambda x: 0.01 * x ** 3 - 0.2 * x ** 2 + x
    df = lambda x: 0.03 * x ** 2 - 0.4 * x + 1
    inner_c, inner_n = slice(4, n - 4), slice(5, n - 4)
    assert np.allclose(sbp1d(2, n, f(xn))[inner_c], f(xc)[inner_c], atol=1e-12)
    assert np.allclose(sbp1d(3, n, f(xc))[inner_n], f(xn)[inner_n], atol=1e-12)
    assert np.allclose(sbp1d(0, n, f(xn))[inner_c], df(xc)[inner_c], atol=1e-12)
    assert np.allclose(sbp1d(1, n, f(xc))[inner_n], df(xn)[inner_n], atol=1e-12)


def test_golden_fixtures_regression(oracle_built):
    """Committed oracle outputs (tests/golden/make_golden.py): a regression pin of the
    restatement itself, not reference output."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "oracle_c8.npz")
    g = np.load(path)
    o = Oracle(8, h_mean=float(g["h_mean"]))
    out = o.apply(g["h"], g["u"], g["v"])
    for a, b in zip(out, (g["dh"], g["du"], g["dv"])):
        assert np.array_equal(a, b)
    r = o.rk4(g["h"], g["u"], g["v"], float(g["dt"]), int(g["nsteps"]))
    for a, b in zip(r, (g["h3"], g["u3"], g["v3"])):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("order", [42, 21, 63])
def test_curl_of_gradient_vanishes(order):
    """curl_ch_sbp_sat_* of the covariant gradient of a smooth field is zero to
    rounding: the i2c differences along x and y commute and the SAT terms vanish
    because both panels hold the same tangential derivative on a shared edge, which
    pins the exchange's orientation signs."""
    o = Oracle(20, sbp_order=order)
    h = o.gaussian(lam0=1.0, phi0=0.4, d0=0.5, amp=1.0)[0]
    gx, gy = o.grad(h)
    c = o.curl(gx, gy)
    scale = max(np.abs(gx).max(), np.abs(gy).max()) / EARTH_RADIUS
    assert np.abs(c).max() < 1e-11 * scale


@pytest.mark.parametrize("order,expect", [(42, 1.8), (21, 1.8), (63, 2.4)])
def test_curl_solid_body_rotation_converges(order, expect):
    """The curl of a solid-body rotation about a tilted axis converges to
    2 u0 / a (r . axis) in the max norm (order 2 with the 4-2 and 2-1 closures, near 3
    with 6-3)."""
    ax = np.array([np.sin(0.7), 0.0, np.cos(0.7)])
    errs = []
    for N in (16, 32, 64):
        o = Oracle(N, sbp_order=order)
        _, u, v = o.ts2(u0=20.0, h_mean=1000.0, axis=ax)
        z = o.curl(u, v)
        r = np.stack([o.metric(3, w) for w in (5, 6, 7)])
        ex = 2 * 20.0 / EARTH_RADIUS * np.tensordot(ax, r, 1)
        errs.append(np.abs(z - ex).max() / np.abs(ex).max())
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert rates.min() > expect, (errs, rates)


def test_energies_consistent_across_orders():
    """calc_energies of a smooth state agrees between the SBP orders to their
    truncation error, and PE is g/2 <h, h>."""
    ax = (0.3, 0.0, 0.95)
    vals = {}
    for order in (21, 42, 63):
        o = Oracle(48, h_mean=3000.0, axis=ax, sbp_order=order)
        h, u, v = o.ts2(u0=30.0, h_mean=3000.0, axis=ax)
        vals[order] = np.array(o.energies(h, u, v))
        assert abs(vals[order][2] - 0.5 * EARTH_GRAV * o.dot(0, h, h)) < 1e-13 * vals[order][2]
        assert abs(vals[order][0] - vals[order][1] - vals[order][2]) < 1e-13 * vals[order][0]
    assert np.all(np.abs(vals[42] - vals[63]) < 1e-5 * np.abs(vals[63]))
    assert np.all(np.abs(vals[21] - vals[63]) < 1e-3 * np.abs(vals[63]))


def test_latlon_regrid_converges():
    """The oracle's cubic lat-lon regrid of a smooth xy field (through the ECS_xy halo of
    width 2) converges at fourth order and reads no unfilled halo value."""
    errs = []
    for N in (16, 32, 64):
        o = Oracle(N)
        h = o.gaussian(lam0=1.0, phi0=0.4, d0=0.5, amp=1.0)[0]
        ll = o.latlon(h)
        nlat, nlon = ll.shape
        assert (nlat, nlon) == (2 * N + 1, 4 * N) and not np.isnan(ll).any()
        phi = -np.pi / 2 + np.arange(nlat) * np.pi / (nlat - 1)
        lam = np.arange(nlon) * 2 * np.pi / nlon
        P, L = np.meshgrid(phi, lam, indexing="ij")
        c0 = (np.cos(0.4) * np.cos(1.0), np.cos(0.4) * np.sin(1.0), np.sin(0.4))
        d = np.clip(np.cos(P) * np.cos(L) * c0[0] + np.cos(P) * np.sin(L) * c0[1] + np.sin(P) * c0[2], -1, 1)
        errs.append(np.abs(ll - np.exp(-(np.arccos(d) / 0.5) ** 2)).max())
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert rates.min() > 3.5, (errs, rates)


def _ah_w2(N, u0, axis):
    from ch_swe_b200.testcases import williamson2
    h, u, v = williamson2(N, u0=u0, h_mean=0.0, axis=axis, linear_mode=True, staggering="Ah")
    return h, u, v


@pytest.mark.parametrize("order", [42, 21, 63])
def test_ah_operator_pins(order):
    """Ah staggering (node SBP 4-2 with projections): the gradient of a constant
    vanishes, RK4 conserves mass to round-off, and the energy error falls as dt^5,
    i.e. the semi-discrete energy is conserved (a sign or swap error in the vector
    or scalar projection breaks that)."""
    from ch_swe_b200.testcases import gaussian_hill
    N = 16
    o = Oracle(N, h_mean=1000.0, axis=(0.2, 0.1, 0.97), sbp_order=order)
    h, u, v = gaussian_hill(N, 1.0, 0.3, 0.3, 10.0, staggering="Ah")
    dh, du, dv = o.ah_apply(np.ones_like(h), 0 * u, 0 * v)
    assert np.abs(du).max() < 1e-18 and np.abs(dv).max() < 1e-18
    m0, e0 = o.ah_integrals(h, u, v)
    drift = []
    for dt in (600.0, 300.0):
        hs, us, vs = o.ah_rk4(h, u, v, dt, int(14400 / dt))
        m1, e1 = o.ah_integrals(hs, us, vs)
        assert abs(m1 - m0) < 1e-13 * abs(m0)
        drift.append(abs(e1 - e0) / e0)
    assert drift[0] < 1e-7 and drift[0] / drift[1] > 20


@pytest.mark.parametrize("order,expect", [(42, 1.7), (21, 0.9), (63, 2.4)])
def test_ah_williamson2_converges(order, expect):
    """The linear Williamson-2 state is steady for the Ah operator up to a truncation
    error that falls at the order of the node SBP closures (1, 2, 3)."""
    axis = (np.sin(0.6), 0.0, np.cos(0.6))
    u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
    errs = []
    for N in (16, 32, 64):
        o = Oracle(N, h_mean=29400 / EARTH_GRAV, axis=axis, sbp_order=order)
        h, u, v = _ah_w2(N, u0, axis)
        dh, du, dv = o.ah_apply(h, u, v)
        errs.append(max(np.abs(dh).max() / np.abs(h).max(), np.abs(du).max() / np.abs(u).max()))
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert rates.min() > expect, (errs, rates)


def test_latlon_wind_regrid_converges():
    """The oracle's wind regrid (Ch to vertex interpolation, covariant ecs_xy_vec halo
    with its transform matrices, rotation to lat-lon components) converges to the
    exact wind of a solid-body rotation about a tilted axis, away from the poles; a
    wrong transform matrix or rotation leaves an O(1) error."""
    ax = np.array([np.sin(0.7), 0.0, np.cos(0.7)])
    u0 = 20.0
    errs = []
    for N in (16, 32, 64):
        o = Oracle(N)
        _, u, v = o.ts2(u0=u0, h_mean=1000.0, axis=ax)
        uo, vo = o.latlon_vec(u, v)
        nlat, nlon = uo.shape
        assert not np.isnan(uo).any() and not np.isnan(vo).any()
        phi = -np.pi / 2 + np.arange(nlat) * np.pi / (nlat - 1)
        lam = np.arange(nlon) * 2 * np.pi / nlon
        P, L = np.meshgrid(phi, lam, indexing="ij")
        r = np.stack([np.cos(P) * np.cos(L), np.cos(P) * np.sin(L), np.sin(P)], -1)
        vel = u0 * np.cross(ax, r)
        iv = np.stack([-np.sin(L), np.cos(L), 0 * L], -1)
        jv = np.stack([-np.sin(P) * np.cos(L), -np.sin(P) * np.sin(L), np.cos(P)], -1)
        inner = slice(1, nlat - 1)
        errs.append(max(np.abs(uo - (vel * iv).sum(-1))[inner].max(), np.abs(vo - (vel * jv).sum(-1))[inner].max()))
    assert errs[0] < 5e-3 * u0
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert rates.min() > 1.7, (errs, rates)
