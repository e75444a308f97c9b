"""The oracle's diffusion on the Ah staggering (laplace_Ah_sbp{21,42,63}_narrow,
hordiff_scalar_Ah_sbp_*_narrow, hordiff_vec_xyz_Ah_sbp_*_narrow,
explicit_Eul1), pinned by properties that a wrong metric factor, closure coefficient,
penalty sign, stencil offset or sync order breaks: the narrow SBP Laplacian is
self-adjoint and negative semi-definite in the J-weighted SBP node quadrature of its
order and conserves mass (continuous fields: the duplicated panel-edge vertices
agree), kills constants, and converges to the spherical Laplacian (2-1: second order
inside the panels, first order on their edges, an O(1) error of the panel-wise operator
at the cube corners; 4-2: second order in L2, first order on the edges and corners;
6-3: about third order in L2, second order in the max-norm);
the scalar tendency is -(c a hx)^4 L(L(h)); the wind's follows the Cartesian
components; one Euler step is v + dt tendency."""
import numpy as np
import pytest

from oracle.oracle import EARTH_RADIUS, Oracle

A = EARTH_RADIUS


def smooth_field(o, seed):
    """A random smooth function of the position: equal on the duplicated vertices."""
    rng = np.random.default_rng(seed)
    x, y, z = o.metric(0, 5), o.metric(0, 6), o.metric(0, 7)
    f = np.zeros_like(x)
    for _ in range(4):
        k = rng.normal(size=3) * 2.0
        f += rng.normal() * np.sin(k[0] * x + k[1] * y + k[2] * z + rng.uniform(0, 2 * np.pi))
    return f


H63 = [0.3159490740740741, 1.3903935185185186, 0.6275462962962963, 1.2405092592592593, 0.9116898148148148,
       1.0139120370370371]   # the 6-3 node norm (sbp_operators_collection_mod.f90:38-40)


def quad_weights(o, order=21):
    """J times the node norm: Q21_A, Q42_A, Q63_A (sbp_operators_collection_mod.f90:22,35,38-40)."""
    n = o.N + 1
    w1 = np.ones(n)
    edge = {21: [0.5], 42: [17 / 48, 59 / 48, 43 / 48, 49 / 48], 63: H63}[order]
    for i, v in enumerate(edge):
        w1[i] = w1[-1 - i] = v
    return o.metric(0, 0) * w1[None, :, None] * w1[None, None, :]


@pytest.fixture(scope="module")
def orc(oracle_built):
    return Oracle(16)


@pytest.mark.parametrize("order", [21, 42, 63])
def test_laplacian_kills_constants(order, oracle_built):
    o = Oracle(17)
    L = o.lap_ah(np.full((6, 18, 18), 7.5), order)
    assert np.abs(L).max() * A * A / 7.5 < 1e-9


@pytest.mark.parametrize("order,N", [(21, 8), (21, 13), (21, 16), (42, 12), (42, 16), (42, 23), (63, 17), (63, 24),
                                     (63, 33)])
def test_laplacian_self_adjoint_negative_and_conservative(order, N, oracle_built):
    o = Oracle(N)
    w = quad_weights(o, order)
    f, g = smooth_field(o, 1), smooth_field(o, 2)
    Lf, Lg = o.lap_ah(f, order), o.lap_ah(g, order)
    s1, s2 = (w * g * Lf).sum(), (w * f * Lg).sum()
    assert abs(s1 - s2) / abs(s1) < 1e-12
    assert abs((w * Lf).sum()) / np.abs(w * Lf).sum() < 1e-12
    assert (w * f * Lf).sum() < 0 and (w * g * Lg).sum() < 0


def test_laplacian_converges_to_spherical_laplacian(oracle_built):
    err = {}
    for N in (16, 32):
        o = Oracle(N)
        z = o.metric(0, 7)
        e = (o.lap_ah(z) + 2.0 / A ** 2 * z) / (2.0 / A ** 2)
        inner = np.abs(e[:, 1:-1, 1:-1]).max()
        edges = np.abs(np.concatenate([e[:, 0, 1:-1].ravel(), e[:, -1, 1:-1].ravel(),
                                       e[:, 1:-1, 0].ravel(), e[:, 1:-1, -1].ravel()])).max()
        err[N] = (inner, edges)
    assert err[32][0] / err[16][0] < 0.3      # second order inside the panels
    assert err[32][1] / err[16][1] < 0.6      # first order on the panel edges
    assert err[32][0] < 1e-3


def test_laplacian42_converges(oracle_built):
    err = {}
    for N in (16, 32):
        o = Oracle(N)
        z = o.metric(0, 7)
        e = (o.lap_ah(z, 42) + 2.0 / A ** 2 * z) / (2.0 / A ** 2)
        err[N] = (np.sqrt((e ** 2).mean()), np.abs(e).max())
    assert err[32][0] / err[16][0] < 0.35     # second order in L2
    assert err[32][1] / err[16][1] < 0.6      # first order at the edges and corners
    assert err[32][1] < 0.05


def test_laplacian63_converges(oracle_built):
    err = {}
    for N in (24, 48):
        o = Oracle(N)
        z = o.metric(0, 7)
        e = (o.lap_ah(z, 63) + 2.0 / A ** 2 * z) / (2.0 / A ** 2)
        err[N] = (np.sqrt((e ** 2).mean()), np.abs(e).max())
    assert err[48][0] / err[24][0] < 0.2      # about third order in L2
    assert err[48][1] / err[24][1] < 0.35     # second order in the max-norm
    assert err[48][1] < 5e-3


def test_scalar_diffusion_is_minus_c4_bilaplacian(orc):
    o = orc
    h = smooth_field(o, 5) * 100.0
    c = 0.01
    dh, du, dv = o.diff_apply(h, np.zeros_like(h), np.zeros_like(h), uv_coeff=0.03, h_coeff=c)
    dc = c * A * (0.5 * np.pi / o.N)
    want = -1.0 * ((dc * dc) * (dc * dc)) * o.lap_ah(o.lap_ah(h))
    assert np.abs(dh - want).max() <= 1e-14 * np.abs(want).max()
    assert np.abs(du).max() == 0.0 and np.abs(dv).max() == 0.0


def test_vector_diffusion_of_solid_rotation(oracle_built):
    """The Cartesian components of a solid rotation are first-degree harmonics: L(L(V)) =
    4 V / a^4 up to discretisation error, so (du, dv) -> -4 (c hx)^4 (V.b1, V.b2), and
    V.b1 = Qi11 u + Qi12 v, V.b2 = Qi12 u + Qi22 v for covariant (u, v)."""
    from ch_swe_b200.testcases import williamson2
    err = []
    for N in (16, 32):
        o = Oracle(N)
        h, u, v = williamson2(N, staggering="Ah")
        c = 0.03
        _, du, dv = o.diff_apply(h, u, v, uv_coeff=c, h_coeff=0.0)
        k = -4.0 * (c * 0.5 * np.pi / N) ** 4
        Q1, Q2, Q3 = o.metric(0, 1), o.metric(0, 2), o.metric(0, 3)
        wu, wv = k * (Q1 * u + Q2 * v), k * (Q2 * u + Q3 * v)
        s = max(np.abs(wu).max(), np.abs(wv).max())
        err.append(max(np.abs(du - wu)[:, 2:-2, 2:-2].max(), np.abs(dv - wv)[:, 2:-2, 2:-2].max()) / s)
    assert err[1] < 0.05 and err[1] / err[0] < 0.6


def test_euler_step_is_state_plus_dt_tendency(orc):
    o = orc
    rng = np.random.default_rng(9)
    st = tuple(smooth_field(o, s) * m + 0.01 * rng.standard_normal((6, 17, 17)) for s, m in ((11, 50.0), (12, 10.0),
                                                                                                (13, 10.0)))
    t = o.diff_apply(*st, uv_coeff=0.03, h_coeff=0.01)
    out = o.diff_step(*st, dt=600.0, uv_coeff=0.03, h_coeff=0.01, nsteps=1)
    for a, x, d in zip(out, st, t):
        assert np.array_equal(a, x + 600.0 * d)


def test_other_orders_refused(orc, oracle_built):
    with pytest.raises(ValueError):
        orc.diff_apply(*(np.zeros((6, 17, 17)),) * 3, uv_coeff=0.0, h_coeff=0.0, lap_order=43)
    with pytest.raises(ValueError):   # 4-2's closure blocks overlap below N = 11
        Oracle(10).diff_apply(*(np.zeros((6, 11, 11)),) * 3, uv_coeff=0.0, h_coeff=0.0, lap_order=42)
    with pytest.raises(ValueError):   # 6-3's closure blocks overlap below N = 17
        orc.diff_apply(*(np.zeros((6, 17, 17)),) * 3, uv_coeff=0.0, h_coeff=0.0, lap_order=63)
