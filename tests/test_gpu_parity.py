"""GPU parity of the CUDA path (through the C ABI) against the CPU FP64 oracle.

Tolerances: the FP64 device path matches the oracle within 1e-12 relative
(max-norm of the difference over the max-norm of the oracle field); the FP32
path is checked against stated error bounds.
"""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12


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


# tile edges at 1 + 32k (x) and 1 + 16k (y): cover tiles that start at N-2 .. N+1
@pytest.mark.parametrize("N", [8, 12, 15, 16, 17, 18, 24, 31, 32, 33, 34, 35, 47, 48])
def test_apply_parity_fp64_random(N):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    h, u, v = random_state(N, 100 + N)
    o = Oracle(N, h_mean=1000.0)
    ref = o.apply(h, u, v)
    dom = create_domain(N, h_mean=1000.0)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    got = y.download()
    for g, r, name in zip(got, ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (name, rel(g, r))


# every tile size, with tile edges falling next to the closure rows
@pytest.mark.parametrize("tile,N", [(17, 8), (17, 16), (17, 17), (17, 20), (17, 33), (17, 50),
                                    (25, 24), (25, 25), (25, 26), (25, 49), (25, 50),
                                    (33, 20), (33, 66)])
def test_apply_parity_fp64_every_tile(tile, N):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    h, u, v = random_state(N, 300 + N)
    ref = Oracle(N, h_mean=1000.0).apply(h, u, v)
    dom = create_domain(N, h_mean=1000.0)
    dom.tile = tile
    assert dom.tile == tile
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (tile, name, rel(g, r))


KERNEL_CONFIGS = [(t, o, r) for r in (0, 1)
                  for t, o in ((17, 3), (17, 4), (25, 2), (25, 3), (25, 4), (33, 2), (33, 3))]


@pytest.mark.parametrize("cfg", KERNEL_CONFIGS)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_every_kernel_config_matches_oracle(cfg, precision):
    """Every built (tile, blocks-per-SM, runs) configuration: one apply against the oracle."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    N = 26
    h, u, v = random_state(N, 77)
    ref = Oracle(N, h_mean=1000.0).apply(h, u, v)
    dom = create_domain(N, precision=precision, h_mean=1000.0)
    dom.kernel_config = cfg
    assert dom.kernel_config == cfg
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom)
    op.apply(y, x, dom)
    tol = FP64_RTOL if precision == "fp64" else 1e-5
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < tol, (cfg, precision, name, rel(g, r))
    dom.destroy()


@pytest.mark.parametrize("tile", [17, 25, 33])
def test_rk4_every_tile_fp64(tile):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, dt, nst = 24, 900.0, 6
    o = Oracle(N, h_mean=1000.0)
    h, u, v = o.gaussian(lam0=0.7, phi0=0.6, d0=0.2)
    ref = o.rk4(h, u, v, dt, nst)
    dom = create_domain(N, h_mean=1000.0)
    dom.tile = tile
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, nst)
    for g, r, name in zip(x.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (tile, name, rel(g, r))


def test_autotune_picks_a_built_tile_and_leaves_states_alone():
    from ch_swe_b200 import create_domain, create_stvec_swm
    N = 32
    dom = create_domain(N, precision="fp32")
    h, u, v = random_state(N, 7)
    x = create_stvec_swm(dom).upload(h, u, v)
    times = dom.autotune(nreps=3)
    assert set(times) == {17, 25, 33} and all(t > 0 for t in times.values())
    assert dom.tile == min(times, key=times.get)
    for g, r in zip(x.download(), (h, u, v)):
        assert np.array_equal(g, r.astype(np.float32).astype(np.float64))
    with pytest.raises(Exception):
        dom.tile = 21


@pytest.mark.parametrize("N", [16, 33, 34])
def test_contravariant_parity_fp64(N):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    h, u, v = random_state(N, 200 + N)
    ref = Oracle(N).co2contra(u, v)
    dom = create_domain(N)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom).upload(h, u, v)
    op.contravariant(y, x)
    _, ut, vt = y.download()
    assert rel(ut, ref[0]) < FP64_RTOL
    assert rel(vt, ref[1]) < FP64_RTOL


def test_apply_parity_coriolis_constant_tilted_axis():
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    from oracle.oracle import Oracle
    N = 16
    h, u, v = random_state(N, 7)
    for cc, axis in ((True, (0.0, 0.0, 1.0)), (False, (0.3, -0.5, 0.8))):
        o = Oracle(N, h_mean=500.0, omega=1e-4, axis=axis, coriolis_constant=cc)
        ref = o.apply(h, u, v)
        dom = create_domain(N, h_mean=500.0, omega=1e-4, rotation_axis=axis, coriolis_constant=cc)
        op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 500.0}, dom)
        x = create_stvec_swm(dom).upload(h, u, v)
        y = create_stvec_swm(dom)
        op.apply(y, x, dom)
        for g, r, name in zip(y.download(), ref, "huv"):
            assert rel(g, r) < FP64_RTOL, (cc, name, rel(g, r))


def test_rk4_c32_gaussian_96_steps_fp64():
    """Config 1: C32, dt = 900 s, 96 steps, Gaussian hill d0 = 0.15 at a seeded centre."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, dt, nsteps = 32, 900.0, 96
    rng = np.random.default_rng(20261204)
    lam0, phi0 = rng.uniform(0, 2 * np.pi), np.arcsin(rng.uniform(-1, 1))
    o = Oracle(N, h_mean=1000.0)
    h0, u0, v0 = o.gaussian(lam0=lam0, phi0=phi0, d0=0.15)
    ref = o.rk4(h0, u0, v0, dt, nsteps)
    dom = create_domain(N, h_mean=1000.0)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    st = create_stvec_swm(dom).upload(h0, u0, v0)
    ts = create_timescheme(st, "rk4")
    ts.steps(st, op, dom, dt, nsteps)
    got = st.download()
    for g, r, name in zip(got, ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (name, rel(g, r))
        assert rel_l2(g, r) < FP64_RTOL, (name, rel_l2(g, r))
    m_ref, e_ref = o.integrals(*ref)
    m, e = op.integrals(st)
    assert abs(m - m_ref) <= 1e-12 * abs(m_ref)
    assert abs(e - e_ref) <= 1e-12 * abs(e_ref)


def test_rk4_step_matches_steps_and_oracle():
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N = 20
    o = Oracle(N)
    h0, u0, v0 = o.gaussian(lam0=0.3, phi0=0.2, d0=0.3)
    ref = o.rk4(h0, u0, v0, 1200.0, 3)
    dom = create_domain(N)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    a = create_stvec_swm(dom).upload(h0, u0, v0)
    b = create_stvec_swm(dom).upload(h0, u0, v0)
    ts = create_timescheme(a, "rk4")
    for _ in range(3):
        ts.step(a, op, dom, 1200.0)
    ts.steps(b, op, dom, 1200.0, 3)
    ga, gb = a.download(), b.download()
    for x, y, r in zip(ga, gb, ref):
        assert np.array_equal(x, y)
        assert rel(x, r) < FP64_RTOL


def test_fp32_c32_error_bounds():
    """FP32 stencils with Kahan-compensated state: relative L2 error vs the FP64 oracle."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, dt, nsteps = 32, 900.0, 96
    o = Oracle(N, h_mean=1000.0)
    h0, u0, v0 = o.gaussian(lam0=np.pi / 4, phi0=np.arcsin(1 / np.sqrt(3)), d0=0.15)
    ref = o.rk4(h0, u0, v0, dt, nsteps)
    dom = create_domain(N, precision="fp32", h_mean=1000.0)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    st = create_stvec_swm(dom).upload(h0, u0, v0)
    create_timescheme(st, "rk4").steps(st, op, dom, dt, nsteps)
    h, u, v = st.download()
    assert rel_l2(h, ref[0]) < 1e-5, rel_l2(h, ref[0])
    assert rel_l2(u, ref[1]) < 1e-4, rel_l2(u, ref[1])
    assert rel_l2(v, ref[2]) < 1e-4, rel_l2(v, ref[2])


def test_members_are_independent():
    """Several members in one launch give the single-member results bit for bit."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, M = 16, 3
    o = Oracle(N)
    Hs = [600.0, 1000.0, 1700.0]
    ics = [o.gaussian(lam0=0.5 * k, phi0=0.1 * k, d0=0.2 + 0.05 * k, amp=1.0 + k) for k in range(M)]
    dom = create_domain(N, n_members=M)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    for k in range(M):
        op.set_member_h_mean(k, Hs[k])
    st = create_stvec_swm(dom)
    for k in range(M):
        st.upload(*ics[k], member=k)
    create_timescheme(st, "rk4").steps(st, op, dom, 900.0, 5)
    for k in range(M):
        d1 = create_domain(N, h_mean=Hs[k])
        op1 = create_swm_operator(d1.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": Hs[k]}, d1)
        s1 = create_stvec_swm(d1).upload(*ics[k])
        create_timescheme(s1, "rk4").steps(s1, op1, d1, 900.0, 5)
        for a, b in zip(st.download(member=k), s1.download()):
            assert np.array_equal(a, b)
        ref = Oracle(N, h_mean=Hs[k]).rk4(*ics[k], 900.0, 5)
        for a, r in zip(st.download(member=k), ref):
            assert rel(a, r) < FP64_RTOL


def test_stvec_algebra():
    from ch_swe_b200 import create_domain, create_stvec_swm
    N = 9
    dom = create_domain(N)
    a_h = random_state(N, 1)
    b_h = random_state(N, 2)
    c_h = random_state(N, 3)
    a = create_stvec_swm(dom).upload(*a_h)
    b = create_stvec_swm(dom).upload(*b_h)
    c = create_stvec_swm(dom).upload(*c_h)
    c.assign(2.0, a, -0.5, b)
    for g, x, y in zip(c.download(), a_h, b_h):
        assert np.allclose(g, 2.0 * x - 0.5 * y, rtol=1e-15, atol=1e-15)
    c.update(0.25, a, 3.0, b)
    for g, x, y in zip(c.download(), a_h, b_h):
        assert np.allclose(g, 2.0 * x - 0.5 * y + 0.25 * x + 3.0 * y, rtol=1e-14, atol=1e-14)
    c.assign(1.5, a)
    for g, x in zip(c.download(), a_h):
        assert np.array_equal(g, 1.5 * x)


def test_mass_conserved_and_energy_drift_fp64():
    """Mass <h,1> is conserved to round-off; the RK4 energy drift is tiny and reported."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N = 24
    o = Oracle(N)
    h0, u0, v0 = o.gaussian(lam0=1.0, phi0=0.5, d0=0.2)
    dom = create_domain(N)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    st = create_stvec_swm(dom).upload(h0, u0, v0)
    m0, e0 = op.integrals(st)
    create_timescheme(st, "rk4").steps(st, op, dom, 600.0, 50)
    m1, e1 = op.integrals(st)
    assert abs(m1 - m0) < 1e-12 * abs(m0)
    assert abs(e1 - e0) < 1e-6 * abs(e0)


def test_launch_count_reported():
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    dom = create_domain(12)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    st = create_stvec_swm(dom).upload(*random_state(12, 5))
    n0 = dom.launch_count()
    create_timescheme(st, "rk4").steps(st, op, dom, 100.0, 4)
    dom.synchronize()
    assert dom.launch_count() - n0 == 4 * 12
