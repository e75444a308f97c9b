"""GPU parity of the advective operator (advective_swm_operator, covariant Ch:
up4 mass flux, up4 vector advection, Christoffel terms) against the CPU oracle.
FP64: within 1e-12 relative (max-norm over the field's max-norm), for states whose
duplicated panel-edge copies disagree as well as for smooth ones."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
G = 9.80616
H0 = 29400 / G


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built, oracle_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


def rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def random_state(N, seed):
    from ch_swe_b200 import state_shapes
    rng = np.random.default_rng(seed)
    h, u, v = (rng.standard_normal(s) for s in state_shapes(N))
    return H0 + 50.0 * h, 10.0 * u, 10.0 * v


def smooth_state(o, seed):
    rng = np.random.default_rng(seed)
    axis = rng.standard_normal(3)
    axis /= np.linalg.norm(axis)
    h, u, v = o.ts2(u0=30.0, h_mean=H0, axis=axis)
    h = h + o.gaussian(lam0=1.0, phi0=0.4, d0=0.3, amp=40.0)[0]
    return h, u, v


def gpu_apply(N, state, precision="fp64", tile=None, axis=(0.0, 0.0, 1.0), runs=0):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    dom = create_domain(N, precision=precision, operator="advective", rotation_axis=axis)
    if tile:
        dom.kernel_config = (tile, 3 if tile == 17 else 2, runs)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
    x = create_stvec_swm(dom).upload(*state)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    out = y.download()
    dom.destroy()
    return out


@pytest.mark.parametrize("N", [8, 12, 16, 17, 24, 33])
def test_apply_parity_fp64_random(N):
    from oracle.oracle import Oracle
    st = random_state(N, 500 + N)
    ref = Oracle(N, h_mean=H0, operator="advective").apply(*st)
    got = gpu_apply(N, st)
    for g, r, name in zip(got, ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (N, name, rel(g, r))


@pytest.mark.parametrize("runs", [0, 1])
@pytest.mark.parametrize("tile", [17, 25, 33])
def test_apply_parity_fp64_smooth_every_tile(tile, runs):
    """Every built advective stage configuration (tile, with and without stencil runs)."""
    from oracle.oracle import Oracle
    N = 26
    o = Oracle(N, h_mean=H0, operator="advective")
    st = smooth_state(o, 7)
    ref = o.apply(*st)
    got = gpu_apply(N, st, tile=tile, runs=runs)
    for g, r, name in zip(got, ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (tile, runs, name, rel(g, r))


def test_rk4_williamson2_tilted_fp64_matches_oracle():
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import EARTH_RADIUS, Oracle
    N, dt, nst = 20, 1200.0, 8
    axis = (np.sin(0.8), 0.0, np.cos(0.8))
    u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
    o = Oracle(N, h_mean=H0, axis=axis, operator="advective")
    st = o.ts2(u0=u0, h_mean=H0, axis=axis)
    ref = o.rk4(*st, dt, nst)
    dom = create_domain(N, operator="advective", rotation_axis=axis)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
    x = create_stvec_swm(dom).upload(*st)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, nst)
    for g, r, name in zip(x.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (name, rel(g, r))
    dom.destroy()


def test_members_independent_advective():
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    N, M, dt = 16, 3, 1200.0
    states = [random_state(N, 900 + k) for k in range(M)]
    dom = create_domain(N, n_members=M, operator="advective")
    op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
    x = create_stvec_swm(dom)
    for k, s in enumerate(states):
        x.upload(*s, member=k)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, 3)
    for k, s in enumerate(states):
        d1 = create_domain(N, operator="advective")
        op1 = create_swm_operator(d1.grav, {"swm_operator_type": "advective_swm_operator"}, d1)
        x1 = create_stvec_swm(d1).upload(*s)
        create_timescheme(x1, "rk4").steps(x1, op1, d1, dt, 3)
        for a, b in zip(x.download(member=k), x1.download()):
            assert rel(a, b) < 1e-14
        d1.destroy()
    dom.destroy()


def test_fp32_williamson2_against_fp64():
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import EARTH_RADIUS, Oracle
    N, dt, nst = 32, 900.0, 48
    axis = (np.sin(0.5), 0.0, np.cos(0.5))
    u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
    st = Oracle(N, h_mean=H0, axis=axis, operator="advective").ts2(u0=u0, h_mean=H0, axis=axis)
    out = {}
    for prec in ("fp64", "fp32"):
        dom = create_domain(N, precision=prec, operator="advective", rotation_axis=axis)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
        x = create_stvec_swm(dom).upload(*st)
        create_timescheme(x, "rk4").steps(x, op, dom, dt, nst)
        out[prec] = x.download()
        dom.destroy()
    for a, b, name in zip(out["fp32"], out["fp64"], "huv"):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5, name
    # steady state: the FP64 run stays near the analytic state (discretisation error)
    assert rel(out["fp64"][0], st[0]) < 1e-4


@pytest.mark.parametrize("order,N", [(21, 12), (21, 24), (63, 16), (63, 26)])
def test_apply_parity_fp64_sbp_orders(order, N):
    """The advective operator with the SBP 2-1 / 6-3 Ch operators (the _21 / _63 names
    of its div, grad, Coriolis, co2contra and quadrature; the vector advection keeps
    its _sbp42 interpolators, as in the reference) against the oracle."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    st = random_state(N, 40 + N + order)
    ref = Oracle(N, h_mean=H0, operator="advective", sbp_order=order).apply(*st)
    dom = create_domain(N, operator="advective", sbp_order=order)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator",
                                        "div_op_name": f"div_ch_sbp_sat_{order}_proj"}, dom)
    x = create_stvec_swm(dom).upload(*st)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (order, N, name, rel(g, r))
    dom.destroy()


@pytest.mark.parametrize("order", [21, 63])
def test_rk4_williamson2_tilted_sbp_orders(order):
    """Eight RK4 steps of tilted-axis Williamson-2 with the 2-1 / 6-3 operators: FP64
    within 1e-12 of the oracle for every tile, FP32 within 1e-5 of FP64."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import EARTH_RADIUS, Oracle
    N, dt, nst = 20, 1200.0, 8
    axis = (np.sin(0.8), 0.0, np.cos(0.8))
    u0 = 2 * np.pi * EARTH_RADIUS / (12 * 86400)
    o = Oracle(N, h_mean=H0, axis=axis, operator="advective", sbp_order=order)
    st = o.ts2(u0=u0, h_mean=H0, axis=axis)
    ref = o.rk4(*st, dt, nst)
    out = {}
    for prec, tile in (("fp64", 17), ("fp64", 25), ("fp64", 33), ("fp32", 25)):
        dom = create_domain(N, precision=prec, operator="advective", rotation_axis=axis, sbp_order=order)
        dom.kernel_config = (tile, 3 if tile == 17 else 2, 0)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
        x = create_stvec_swm(dom).upload(*st)
        create_timescheme(x, "rk4").steps(x, op, dom, dt, nst)
        out[(prec, tile)] = x.download()
        dom.destroy()
    for tile in (17, 25, 33):
        for g, r, name in zip(out[("fp64", tile)], ref, "huv"):
            assert rel(g, r) < FP64_RTOL, (order, tile, name, rel(g, r))
    for a, b, name in zip(out[("fp32", 25)], out[("fp64", 25)], "huv"):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5, name


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_williamson5_orography_matches_oracle(precision):
    """The advective operator with orography (Williamson test 5: h_total = h + h_surf in
    the gradient, operator_adv_swm_mod.f90:78): applies and RK4 steps against the oracle
    with the same h_surf; without the orography the tendency differs at O(1)."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from ch_swe_b200.testcases import Ts5Orography, williamson5
    from oracle.oracle import Oracle
    N = 24
    h0, u0, v0, hs = williamson5(N)
    # applies on an unbalanced state (the balanced one leaves a tendency of the size of the
    # truncation error, a residual of terms 1e4 times larger)
    rng = np.random.default_rng(55)
    h, u, v = (x + s * rng.standard_normal(x.shape) for x, s in ((h0, 20.0), (u0, 2.0), (v0, 2.0)))
    o = Oracle(N, h_mean=5960.0, operator="advective")
    o.set_orography(hs)
    ref = o.apply(h, u, v)
    dom = create_domain(N, precision=precision, operator="advective")
    op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom,
                             orography_generator=Ts5Orography())
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    tol = FP64_RTOL if precision == "fp64" else 1e-5
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < tol, (name, rel(g, r))
    # the orography matters: without it the wind tendency is another field
    o.set_orography(None)
    flat = o.apply(h, u, v)
    assert rel(flat[1], ref[1]) > 1e-3
    if precision == "fp64":
        ref4 = Oracle(N, h_mean=5960.0, operator="advective")
        ref4.set_orography(hs)
        r4 = ref4.rk4(h0, u0, v0, 900.0, 4)
        x.upload(h0, u0, v0)
        create_timescheme(x, "rk4").steps(x, op, dom, 900.0, 4)
        for g, r, name in zip(x.download(), r4, "huv"):
            assert rel(g, r) < FP64_RTOL, ("rk4", name, rel(g, r))
        # removing it again gives the operator without orography
        op.set_orography(None)
        x.upload(h, u, v)
        op.apply(y, x, dom)
        for g, r, name in zip(y.download(), flat, "huv"):
            assert rel(g, r) < FP64_RTOL, ("none", name, rel(g, r))
    dom.destroy()
