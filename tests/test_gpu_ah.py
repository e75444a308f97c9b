"""GPU parity of the linear operator on the Ah staggering (h, u, v on the cell vertices;
div_ah_sbp_proj_42, grad_ah_sbp_proj_42, coriolis_colocated, co2contra_colocated,
SBP_Ah42_quadrature) against the CPU oracle.  FP64: within 1e-12 relative (max-norm
over the field's max-norm), for random states whose duplicated panel-edge copies
disagree as well as for smooth ones; FP32 against FP64 in relative L2."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
H = 1000.0


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built, oracle_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


def rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def random_state(N, seed):
    rng = np.random.default_rng(seed)
    return tuple(rng.standard_normal((6, N + 1, N + 1)) * s for s in (1.0, 10.0, 10.0))


def ah_domain(N, precision="fp64", members=1, axis=(0.0, 0.0, 1.0), order=42):
    from ch_swe_b200 import create_domain, create_swm_operator
    dom = create_domain(N, precision=precision, horizontal_staggering="Ah", n_members=members, h_mean=H,
                        rotation_axis=axis, sbp_order=order)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": H,
                                        "div_op_name": f"div_ah_sbp_proj_{order}",
                                        "grad_op_name": f"grad_ah_sbp_proj_{order}",
                                        "coriolis_op_name": "coriolis_colocated",
                                        "co2contra_op_name": "co2contra_colocated",
                                        "quadrature_name": f"SBP_Ah{order}_quadrature"}, dom)
    return dom, op


@pytest.mark.parametrize("order,N", [(42, 8), (42, 12), (42, 17), (42, 24), (42, 33), (21, 8), (21, 17),
                                     (63, 16), (63, 25)])
def test_apply_parity_fp64_random(order, N):
    from ch_swe_b200 import create_stvec_swm
    from oracle.oracle import Oracle
    st = random_state(N, 300 + N)
    ref = Oracle(N, h_mean=H, sbp_order=order).ah_apply(*st)
    dom, op = ah_domain(N, order=order)
    x = create_stvec_swm(dom).upload(*st)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (order, N, name, rel(g, r))
    dom.destroy()


@pytest.mark.parametrize("order", [42, 21, 63])
def test_rk4_parity_fp64_and_fp32(order):
    """24 RK4 steps of a Gaussian hill under a tilted rotation axis: FP64 within 1e-12
    of the oracle, FP32 within 1e-5 (relative L2) of FP64; mass conserved."""
    from ch_swe_b200 import create_stvec_swm, create_timescheme
    from ch_swe_b200.testcases import gaussian_hill
    from oracle.oracle import Oracle
    N, dt, nst = 20, 900.0, 24
    axis = (np.sin(0.7), 0.0, np.cos(0.7))
    st = gaussian_hill(N, lam0=0.5, phi0=0.6, d0=0.3, amp=5.0, staggering="Ah")
    o = Oracle(N, h_mean=H, axis=axis, sbp_order=order)
    ref = o.ah_rk4(*st, dt, nst)
    out = {}
    for prec in ("fp64", "fp32"):
        dom, op = ah_domain(N, prec, axis=axis, order=order)
        x = create_stvec_swm(dom).upload(*st)
        create_timescheme(x, "rk4").steps(x, op, dom, dt, nst)
        out[prec] = x.download()
        if prec == "fp64":
            m0, _ = op.integrals(create_stvec_swm(dom).upload(*st))
            m1, _ = op.integrals(x)
            assert abs(m1 - m0) < 1e-12 * np.abs(st[0]).max() * 4 * np.pi
        dom.destroy()
    for g, r, name in zip(out["fp64"], ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (name, rel(g, r))
    for a, b, name in zip(out["fp32"], out["fp64"], "huv"):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5, name


@pytest.mark.parametrize("order", [42, 21, 63])
def test_integrals_match_oracle(order):
    from ch_swe_b200 import create_stvec_swm
    from oracle.oracle import Oracle
    N = 16
    st = random_state(N, 5)
    o = Oracle(N, h_mean=H, sbp_order=order)
    m_ref, e_ref = o.ah_integrals(*st)
    dom, op = ah_domain(N, order=order)
    m, e = op.integrals(create_stvec_swm(dom).upload(*st))
    assert abs(m - m_ref) < 1e-12 * max(abs(m_ref), 1.0) and abs(e - e_ref) < 1e-12 * abs(e_ref)
    dom.destroy()


def test_members_independent():
    from ch_swe_b200 import create_stvec_swm, create_timescheme
    N, M, dt = 12, 3, 900.0
    states = [random_state(N, 700 + k) for k in range(M)]
    dom, op = ah_domain(N, members=M)
    x = create_stvec_swm(dom)
    for k, s in enumerate(states):
        x.upload(*s, member=k)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, 3)
    for k, s in enumerate(states):
        d1, op1 = ah_domain(N)
        x1 = create_stvec_swm(d1).upload(*s)
        create_timescheme(x1, "rk4").steps(x1, op1, d1, dt, 3)
        for a, b in zip(x.download(member=k), x1.download()):
            assert rel(a, b) < 1e-14
        d1.destroy()
    dom.destroy()


def test_williamson2_steady_state_large_cube():
    """C192 (beyond the oracle's sizes): the linear Williamson-2 state is steady up to
    the SBP 4-2 truncation error, and the discrete mass is conserved to round-off over
    one simulated hour."""
    from ch_swe_b200 import create_stvec_swm, create_timescheme
    from ch_swe_b200.testcases import williamson2
    from oracle.oracle import EARTH_GRAV
    N, dt, nst = 192, 150.0, 24
    axis = (np.sin(0.3), 0.0, np.cos(0.3))
    Hw = 29400.0 / EARTH_GRAV
    u0 = 2 * np.pi * 6371229.0 / (12 * 86400)
    h, u, v = williamson2(N, u0=u0, h_mean=Hw, axis=axis, linear_mode=True, staggering="Ah")
    h = h - Hw
    from ch_swe_b200 import create_domain, create_swm_operator
    dom = create_domain(N, precision="fp64", horizontal_staggering="Ah", h_mean=Hw, rotation_axis=axis)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": Hw}, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    m0, _ = op.integrals(x)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, nst)
    h1, u1, v1 = x.download()
    m1, _ = op.integrals(x)
    assert rel(h1, h) < 1e-4 and rel(u1, u) < 1e-4
    assert abs(m1 - m0) < 1e-10 * np.abs(h).max()
    dom.destroy()
