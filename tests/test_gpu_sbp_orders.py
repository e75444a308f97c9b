"""GPU parity of the SBP 2-1 and 6-3 Ch linear operators (the _sbp_sat_21 / _21 and
_63 names of the reference's factories) against the CPU FP64 oracle with the same
order.

Tolerances as for SBP 4-2: FP64 within 1e-12 relative (max-norm of the
difference over the max-norm of the oracle field), FP32 within 1e-5.
"""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
LIN = {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}


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
    return tuple(rng.standard_normal(s) for s in state_shapes(N))


def gpu_apply(N, state, order, precision="fp64", tile=None):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    dom = create_domain(N, precision=precision, h_mean=1000.0, sbp_order=order)
    if tile:
        dom.tile = tile
    op = create_swm_operator(dom.grav, LIN, dom)
    x = create_stvec_swm(dom).upload(*state)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    out = y.download()
    dom.destroy()
    return out


ORDERS = [21, 63]


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("N", [8, 12, 16, 17, 24, 33, 48])
def test_apply_parity_fp64_random(order, N):
    from oracle.oracle import Oracle
    if order == 63 and N < 16:
        pytest.skip("SBP 6-3 needs N >= 16")
    st = random_state(N, 700 + N)
    ref = Oracle(N, h_mean=1000.0, sbp_order=order).apply(*st)
    for g, r, name in zip(gpu_apply(N, st, order), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (order, N, name, rel(g, r))


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("tile,N", [(17, 16), (17, 33), (25, 24), (25, 49), (33, 32), (33, 65)])
def test_apply_parity_fp64_every_tile(order, tile, N):
    from oracle.oracle import Oracle
    st = random_state(N, 800 + N)
    ref = Oracle(N, h_mean=1000.0, sbp_order=order).apply(*st)
    for g, r, name in zip(gpu_apply(N, st, order, tile=tile), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (order, tile, N, name, rel(g, r))


@pytest.mark.parametrize("order", ORDERS)
def test_apply_fp32_within_bound(order):
    from oracle.oracle import Oracle
    N = 26
    o = Oracle(N, h_mean=1000.0, sbp_order=order)
    st = o.gaussian(lam0=0.9, phi0=0.4, d0=0.25)
    ref = o.apply(*st)
    for g, r, name in zip(gpu_apply(N, st, order, precision="fp32"), ref, "huv"):
        assert rel(g, r) < 1e-5, (order, name, rel(g, r))


@pytest.mark.parametrize("order", ORDERS)
def test_rk4_fp64_matches_oracle_and_conserves_mass(order):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, dt, nst = 24, 900.0, 8
    o = Oracle(N, h_mean=1000.0, sbp_order=order)
    h, u, v = o.gaussian(lam0=0.7, phi0=0.6, d0=0.2)
    ref = o.rk4(h, u, v, dt, nst)
    dom = create_domain(N, h_mean=1000.0, sbp_order=order)
    op = create_swm_operator(dom.grav, LIN, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    m0, e0 = op.integrals(x)
    mr0, er0 = o.integrals(h, u, v)
    assert abs(m0 - mr0) < 1e-12 * abs(mr0) and abs(e0 - er0) < 1e-12 * abs(er0)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, nst)
    for g, r, name in zip(x.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (name, rel(g, r))
    m1, _ = op.integrals(x)
    assert abs(m1 - m0) < 1e-12 * abs(m0)
    dom.destroy()


@pytest.mark.parametrize("order", ORDERS)
def test_orders_differ_and_configs_are_checked(order):
    """The orders give different tendencies on the same state; a 2-1 or 6-3 context
    accepts only its built kernel configurations and the linear operator."""
    from ch_swe_b200 import create_domain, create_swm_operator
    from ch_swe_b200._lib import SweError
    from oracle.oracle import Oracle
    N = 16
    st = random_state(N, 5)
    ref42 = Oracle(N, h_mean=1000.0).apply(*st)
    assert rel(gpu_apply(N, st, order)[0], ref42[0]) > 1e-3
    dom = create_domain(N, h_mean=1000.0, sbp_order=order)
    with pytest.raises(SweError):
        dom.kernel_config = (25, 4, 1)
    dom.kernel_config = (25, 2, 0)
    assert dom.kernel_config == (25, 2, 0)
    times = dom.autotune(nreps=2)
    assert dom.kernel_config in ((17, 3, 0), (25, 2, 0), (33, 2, 0)) and set(times) == {17, 25, 33}
    with pytest.raises(ValueError):
        create_swm_operator(dom.grav, dict(LIN, div_op_name="div_ch_sbp_sat_42_proj"), dom)
    dom.destroy()
