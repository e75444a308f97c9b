"""The fused stage of the linear Ch operator (SBP 4-2) against the CPU FP64 oracle.

The fused stage computes the contravariant components inside the stage kernel from
TMA-loaded tiles, and the edge strips with a kernel of their own.  Tolerances as
for the split kernels: FP64 within 1e-12 relative (max-norm) of the oracle, FP32
within the stated error bounds.  Cube sizes are chosen so that tile edges fall at
every distance from the SBP closure rows, with one, two and several tiles per panel
in both directions.
"""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
LIN = {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}
CFG64 = [(17, 2, 2), (25, 1, 2)]
CFG32 = [(17, 4, 2), (25, 3, 2), (33, 2, 2)]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built, oracle_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


def rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def random_state(N, seed):
    from ch_swe_b200 import state_shapes
    rng = np.random.default_rng(seed)
    return tuple(rng.standard_normal(s) for s in state_shapes(N))


def fused_domain(N, cfg, **kw):
    from ch_swe_b200 import create_domain
    dom = create_domain(N, **kw)
    dom.kernel_config = cfg
    assert dom.kernel_config == cfg
    return dom


@pytest.mark.parametrize("cfg", CFG64)
@pytest.mark.parametrize("N", [8, 12, 16, 17, 20, 24, 25, 26, 27, 33, 38, 40, 49, 52, 64, 77])
def test_fused_apply_parity_fp64(cfg, N):
    from ch_swe_b200 import create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    h, u, v = random_state(N, 500 + N)
    ref = Oracle(N, h_mean=1000.0).apply(h, u, v)
    dom = fused_domain(N, cfg, h_mean=1000.0)
    op = create_swm_operator(dom.grav, LIN, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    dom.synchronize()
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (cfg, N, name, rel(g, r))
    dom.destroy()


@pytest.mark.parametrize("cfg", CFG32)
@pytest.mark.parametrize("N", [26, 50, 64, 96])
def test_fused_apply_fp32(cfg, N):
    from ch_swe_b200 import create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    h, u, v = random_state(N, 77)
    ref = Oracle(N, h_mean=1000.0).apply(h, u, v)
    dom = fused_domain(N, cfg, precision="fp32", h_mean=1000.0)
    op = create_swm_operator(dom.grav, LIN, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    dom.synchronize()
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < 1e-5, (cfg, name, rel(g, r))
    dom.destroy()


def test_fused_apply_tilted_axis_and_constant_coriolis():
    from ch_swe_b200 import create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    N = 30
    h, u, v = random_state(N, 7)
    for cc, axis in ((True, (0.0, 0.0, 1.0)), (False, (0.3, -0.5, 0.8))):
        ref = Oracle(N, h_mean=500.0, omega=1e-4, axis=axis, coriolis_constant=cc).apply(h, u, v)
        dom = fused_domain(N, CFG64[0], h_mean=500.0, omega=1e-4, rotation_axis=axis, coriolis_constant=cc)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 500.0}, dom)
        x = create_stvec_swm(dom).upload(h, u, v)
        y = create_stvec_swm(dom)
        op.apply(y, x, dom)
        for g, r, name in zip(y.download(), ref, "huv"):
            assert rel(g, r) < FP64_RTOL, (cc, name, rel(g, r))
        dom.destroy()


def test_fused_rk4_c32_gaussian_96_steps_fp64():
    """Config 1 (C32, dt 900 s, 96 steps, seeded Gaussian hill d0 = 0.15) through the fused stage."""
    from ch_swe_b200 import create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, dt, nsteps = 32, 900.0, 96
    rng = np.random.default_rng(20261204)
    lam0, phi0 = rng.uniform(0, 2 * np.pi), np.arcsin(rng.uniform(-1, 1))
    o = Oracle(N, h_mean=1000.0)
    ic = o.gaussian(lam0=lam0, phi0=phi0, d0=0.15)
    ref = o.rk4(*ic, dt, nsteps)
    for cfg in CFG64:
        dom = fused_domain(N, cfg, h_mean=1000.0)
        op = create_swm_operator(dom.grav, LIN, dom)
        st = create_stvec_swm(dom).upload(*ic)
        create_timescheme(st, "rk4").steps(st, op, dom, dt, nsteps)
        dom.synchronize()
        for g, r, name in zip(st.download(), ref, "huv"):
            assert rel(g, r) < FP64_RTOL, (cfg, name, rel(g, r))
            assert rel_l2(g, r) < FP64_RTOL, (cfg, name, rel_l2(g, r))
        m_ref, e_ref = o.integrals(*ref)
        m, e = op.integrals(st)
        assert abs(m - m_ref) <= 1e-12 * abs(m_ref)
        assert abs(e - e_ref) <= 1e-12 * abs(e_ref)
        dom.destroy()


def test_fused_matches_split_fp64():
    """The fused and the split stage agree to rounding over RK4 steps of a smooth state."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from ch_swe_b200.testcases import gaussian_hill
    N = 61
    ic = gaussian_hill(N, lam0=0.4, phi0=0.3, d0=0.2, amp=1.0)
    out = []
    for cfg in [(25, 3, 0), (17, 2, 2), (25, 1, 2)]:
        dom = create_domain(N)
        dom.kernel_config = cfg
        op = create_swm_operator(dom.grav, LIN, dom)
        st = create_stvec_swm(dom).upload(*ic)
        create_timescheme(st, "rk4").steps(st, op, dom, 600.0, 20)
        out.append(st.download())
        dom.destroy()
    for other in out[1:]:
        for a, b, name in zip(other, out[0], "huv"):
            assert rel(a, b) < 1e-13, (name, rel(a, b))


def test_fused_fp32_c32_error_bounds():
    from ch_swe_b200 import create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, dt, nsteps = 32, 900.0, 96
    o = Oracle(N, h_mean=1000.0)
    ic = o.gaussian(lam0=np.pi / 4, phi0=np.arcsin(1 / np.sqrt(3)), d0=0.15)
    ref = o.rk4(*ic, dt, nsteps)
    for cfg in CFG32:
        dom = fused_domain(N, cfg, precision="fp32", h_mean=1000.0)
        op = create_swm_operator(dom.grav, LIN, dom)
        st = create_stvec_swm(dom).upload(*ic)
        create_timescheme(st, "rk4").steps(st, op, dom, dt, nsteps)
        h, u, v = st.download()
        assert rel_l2(h, ref[0]) < 1e-5, (cfg, rel_l2(h, ref[0]))
        assert rel_l2(u, ref[1]) < 1e-4, (cfg, rel_l2(u, ref[1]))
        assert rel_l2(v, ref[2]) < 1e-4, (cfg, rel_l2(v, ref[2]))
        dom.destroy()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fused_members_independent_and_frozen(precision):
    """Members of one launch give the single-member results bit for bit; a member whose
    time step is 0 stays as it was."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, M = 20, 3
    cfg = CFG64[0] if precision == "fp64" else CFG32[0]
    o = Oracle(N)
    Hs = [600.0, 1000.0, 1700.0]
    ics = [o.gaussian(lam0=0.5 * k, phi0=0.1 * k, d0=0.2 + 0.05 * k, amp=1.0 + k) for k in range(M)]
    dom = fused_domain(N, cfg, precision=precision, n_members=M)
    op = create_swm_operator(dom.grav, LIN, dom)
    for k in range(M):
        op.set_member_h_mean(k, Hs[k])
    st = create_stvec_swm(dom)
    for k in range(M):
        st.upload(*ics[k], member=k)
    create_timescheme(st, "rk4").steps(st, op, dom, 900.0, 5)
    for k in range(M):
        d1 = fused_domain(N, cfg, precision=precision, h_mean=Hs[k])
        op1 = create_swm_operator(d1.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": Hs[k]}, d1)
        s1 = create_stvec_swm(d1).upload(*ics[k])
        create_timescheme(s1, "rk4").steps(s1, op1, d1, 900.0, 5)
        for a, b in zip(st.download(member=k), s1.download()):
            assert np.array_equal(a, b)
        d1.destroy()
    before = [st.download(member=k) for k in range(M)]
    create_timescheme(st, "rk4").steps_members(st, op, [600.0, 0.0, 300.0], 3)
    frozen = st.download(member=1)
    for a, b in zip(frozen, before[1]):
        assert np.array_equal(a, b)
    dom.destroy()


def test_fused_configs_selectable_and_rejected_where_not_built():
    from ch_swe_b200 import create_domain
    dom = create_domain(24, precision="fp32")
    for cfg in CFG32:
        dom.kernel_config = cfg
        assert dom.kernel_config == cfg
        assert dom.tile == cfg[0]
    with pytest.raises(Exception):
        dom.kernel_config = (25, 1, 2)        # an FP64 configuration
    dom.kernel_config = (25, 3, 0)
    assert dom.kernel_config == (25, 3, 0)
    dom.destroy()
    adv = create_domain(24, operator="advective")
    with pytest.raises(Exception):
        adv.kernel_config = (25, 3, 2)
    adv.destroy()
