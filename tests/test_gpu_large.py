"""The linear Ch path at the bench's size (C192, the day workload) and at a large
cube (C768), beyond the oracle's sizes: properties that hold whatever the size.
SBP mass conservation to round-off, semi-discrete energy conservation up to the
RK4 error (falling as dt^5), the linear Williamson-2 state staying steady, and
FP32 within 1e-5 (relative L2) of FP64."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


def _run(N, precision, ic, dt, nsteps, h_mean=1000.0, axis=(0.0, 0.0, 1.0)):
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    dom = create_domain(N, precision=precision, h_mean=h_mean, rotation_axis=axis)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": h_mean}, dom)
    x = create_stvec_swm(dom).upload(*ic)
    m0, e0 = op.integrals(x)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, nsteps)
    m1, e1 = op.integrals(x)
    out = x.download()
    dom.destroy()
    return out, (m0, e0), (m1, e1)


def test_c192_day_workload_conservation_and_precision():
    """A sixth of the day workload (C192, cube-corner Gaussian, dt 150 s, 96 steps):
    mass conserved to round-off in FP64, the energy error falls as dt^5, and FP32
    stays within 1e-5 of FP64."""
    from ch_swe_b200.testcases import gaussian_hill
    N = 192
    ic = gaussian_hill(N, lam0=np.pi / 4, phi0=np.arcsin(1 / np.sqrt(3)), d0=0.15, amp=1.0)
    scale = np.abs(ic[0]).sum() * (np.pi / 2 / N) ** 2
    out64, (m0, e0), (m1, e1) = _run(N, "fp64", ic, 150.0, 96)
    assert abs(m1 - m0) < 1e-12 * scale
    _, _, (_, e2) = _run(N, "fp64", ic, 300.0, 48)
    d150, d300 = abs(e1 - e0) / e0, abs(e2 - e0) / e0
    assert d300 < 1e-6 and d300 / max(d150, 1e-300) > 20
    out32, _, _ = _run(N, "fp32", ic, 150.0, 96)
    for a, b, name in zip(out32, out64, "huv"):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5, name


def test_c768_williamson2_steady_and_mass():
    """C768 FP64 (about 85 MB per state box): the linear Williamson-2 state stays steady
    to its truncation error over 8 steps and the mass is conserved to round-off."""
    from ch_swe_b200.testcases import williamson2
    from oracle.oracle import EARTH_GRAV
    N = 768
    Hw = 29400.0 / EARTH_GRAV
    axis = (np.sin(0.4), 0.0, np.cos(0.4))
    u0 = 2 * np.pi * 6371229.0 / (12 * 86400)
    h, u, v = williamson2(N, u0=u0, h_mean=Hw, axis=axis, linear_mode=True)
    ic = (h - Hw, u, v)
    out, (m0, _), (m1, _) = _run(N, "fp64", ic, 37.5, 8, h_mean=Hw, axis=axis)
    for a, b, name in zip(out, ic, "huv"):
        assert np.abs(a - b).max() < 1e-5 * np.abs(b).max(), name
    assert abs(m1 - m0) < 1e-11 * np.abs(ic[0]).sum() * (np.pi / 2 / N) ** 2


def _corner_gaussian(N, seed=20261203 + 1):
    """The day workload's initial state: a Gaussian (d0 = 0.15) on the cube corner with a
    seeded jitter of at most 1e-3 rad."""
    from ch_swe_b200.testcases import gaussian_hill
    rng = np.random.default_rng(seed)
    lam0 = 0.25 * np.pi + rng.uniform(-1e-3, 1e-3)
    phi0 = np.arcsin(1.0 / np.sqrt(3.0)) + rng.uniform(-1e-3, 1e-3)
    return gaussian_hill(N, lam0=lam0, phi0=phi0, d0=0.15, amp=1.0)


@pytest.mark.parametrize("cfg", [(25, 3, 0), (17, 2, 2)])
def test_c192_day_workload_fp64_matches_oracle(cfg):
    """The day workload at its own size (C192, dt 150 s) for 48 RK4 steps: the FP64 GPU
    path, split and fused stage, against the CPU oracle within 1e-12 (max norm and L2)."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import Oracle
    N, dt, nsteps = 192, 150.0, 48
    ic = _corner_gaussian(N)
    ref = Oracle(N, h_mean=1000.0).rk4(*ic, dt, nsteps)
    dom = create_domain(N, h_mean=1000.0)
    dom.kernel_config = cfg
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    x = create_stvec_swm(dom).upload(*ic)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, nsteps)
    dom.synchronize()
    for g, r, name in zip(x.download(), ref, "huv"):
        assert np.abs(g - r).max() < 1e-12 * np.abs(r).max(), (cfg, name)
        assert np.linalg.norm(g - r) < 1e-12 * np.linalg.norm(r), (cfg, name)
    dom.destroy()


def test_c384_advective_williamson2_fp64_matches_oracle():
    """The nonlinear workload at its own size (C384, Williamson 2 about a seeded tilted
    axis, dt 75 s) for 4 RK4 steps: the FP64 GPU advective operator against the CPU
    oracle.  The state is steady, so the change over the steps is compared as well."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    from oracle.oracle import EARTH_GRAV, EARTH_RADIUS, Oracle
    N, dt, nsteps = 384, 75.0, 4
    rng = np.random.default_rng(20261203 + 3)
    theta = float(rng.uniform(0.0, 0.5 * np.pi))
    axis = (np.sin(theta), 0.0, np.cos(theta))
    hm = 2.94e4 / EARTH_GRAV
    u0 = 2.0 * np.pi * EARTH_RADIUS / (12.0 * 86400.0)
    o = Oracle(N, h_mean=hm, axis=axis, operator="advective")
    ic = o.ts2(u0=u0, h_mean=hm, axis=axis)
    ref = o.rk4(*ic, dt, nsteps)
    dom = create_domain(N, operator="advective", rotation_axis=axis)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
    x = create_stvec_swm(dom).upload(*ic)
    create_timescheme(x, "rk4").steps(x, op, dom, dt, nsteps)
    dom.synchronize()
    for g, r, a, name in zip(x.download(), ref, ic, "huv"):
        assert np.abs(g - r).max() < 1e-12 * np.abs(r).max(), name
        dr = r - a
        assert np.abs((g - a) - dr).max() < 1e-8 * np.abs(dr).max(), name
    dom.destroy()
