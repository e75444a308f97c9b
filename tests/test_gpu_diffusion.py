"""GPU parity of the diffusion on the Ah staggering (hordiff_vec_xyz_Ah_sbp_<o>_narrow for
u, v, hordiff_scalar_Ah_sbp_<o>_narrow for h, o = 21, 42 or 63, explicit_Eul1) against the CPU
oracle: FP64 tendencies within 1e-12 relative (max-norm over the field's max-norm) for
random states whose duplicated panel-edge copies disagree, Euler steps and the driver's
RK4-then-diffusion loop likewise; FP32 against FP64 in relative L2; members independent;
non-Ah contexts and unbuilt orders refused."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
H = 1000.0
DIFF = {"hordiff_uv_name": "hordiff_vec_xyz_Ah_sbp_21_narrow", "uv_diff_coeff": 0.03,
        "hordiff_h_name": "hordiff_scalar_Ah_sbp_21_narrow", "h_diff_coeff": 0.01}


def diff_config(order):
    return {**DIFF, "hordiff_uv_name": f"hordiff_vec_xyz_Ah_sbp_{order}_narrow",
            "hordiff_h_name": f"hordiff_scalar_Ah_sbp_{order}_narrow"}


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


def ah_domain(N, precision="fp64", members=1, order=21):
    from ch_swe_b200 import create_domain, create_swm_operator
    dom = create_domain(N, precision=precision, horizontal_staggering="Ah", n_members=members, h_mean=H,
                        sbp_order=order)
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": H,
                                        "div_op_name": f"div_ah_sbp_proj_{order}",
                                        "grad_op_name": f"grad_ah_sbp_proj_{order}",
                                        "coriolis_op_name": "coriolis_colocated",
                                        "co2contra_op_name": "co2contra_colocated",
                                        "quadrature_name": f"SBP_Ah{order}_quadrature"}, dom)
    return dom, op


@pytest.mark.parametrize("order,N", [(21, 8), (21, 12), (21, 17), (21, 24), (21, 33), (42, 11), (42, 12), (42, 17),
                                     (42, 24), (42, 33), (63, 17), (63, 24), (63, 33)])
def test_apply_parity_fp64_random(order, N):
    from ch_swe_b200 import create_stvec_swm, create_swm_diff_operator
    from oracle.oracle import Oracle
    st = random_state(N, 700 + N)
    ref = Oracle(N, h_mean=H).diff_apply(*st, uv_coeff=0.03, h_coeff=0.01, lap_order=order)
    dom, _ = ah_domain(N)
    dif = create_swm_diff_operator(diff_config(order), dom)
    x = create_stvec_swm(dom).upload(*st)
    y = create_stvec_swm(dom)
    dif.apply(y, x, dom)
    for g, r, name in zip(y.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (order, N, name, rel(g, r))
    dom.destroy()


@pytest.mark.parametrize("order", [21, 42, 63])
def test_euler_steps_and_driver_loop_fp64(order):
    """Six driver steps on a Gaussian hill: RK4 of the Ah linear operator of the same SBP
    order, then one explicit_Eul1 diffusion step (shallow_water_mod.f90:112-118)."""
    from ch_swe_b200 import create_stvec_swm, create_swm_diff_operator, create_timescheme
    from ch_swe_b200.testcases import gaussian_hill
    from oracle.oracle import Oracle
    N, dt = 20, 900.0
    st = gaussian_hill(N, lam0=0.5, phi0=0.6, d0=0.3, amp=5.0, staggering="Ah")
    o = Oracle(N, h_mean=H, sbp_order=order)
    ref = st
    for _ in range(6):
        ref = o.ah_rk4(*ref, dt, 1)
        ref = o.diff_step(*ref, dt=dt, uv_coeff=0.03, h_coeff=0.01, lap_order=order)
    dom, op = ah_domain(N, order=order)
    dif = create_swm_diff_operator(diff_config(order), dom)
    x = create_stvec_swm(dom).upload(*st)
    rk, eul = create_timescheme(x, "rk4"), create_timescheme(x, "explicit_Eul1")
    for _ in range(6):
        rk.step(x, op, dom, dt)
        eul.step(x, dif, dom, dt)
    for g, r, name in zip(x.download(), ref, "huv"):
        assert rel(g, r) < FP64_RTOL, (name, rel(g, r))
    dom.destroy()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_diffusion_captured_with_rk4_steps(precision):
    """Domain.set_diffusion: eleven graph-replayed RK4 steps (one graph of eight, three
    single steps), each followed by the diffusion step, give the bits of the step-by-step
    loop; per-member time steps diffuse each member with its own dt and leave a frozen
    member as it was."""
    from ch_swe_b200 import create_stvec_swm, create_swm_diff_operator, create_timescheme
    from ch_swe_b200.testcases import gaussian_hill
    N, dt = 20, 900.0
    st = gaussian_hill(N, lam0=0.5, phi0=0.6, d0=0.3, amp=5.0, staggering="Ah")
    a, opa = ah_domain(N, precision, order=42)
    b, opb = ah_domain(N, precision, order=42)
    dif_a, dif_b = create_swm_diff_operator(diff_config(42), a), create_swm_diff_operator(diff_config(42), b)
    xa, xb = create_stvec_swm(a).upload(*st), create_stvec_swm(b).upload(*st)
    a.set_diffusion(dif_a)
    create_timescheme(xa, "rk4").steps(xa, opa, a, dt, 11)
    rk, eul = create_timescheme(xb, "rk4"), create_timescheme(xb, "explicit_Eul1")
    for _ in range(11):
        rk.step(xb, opb, b, dt)
        eul.step(xb, dif_b, b, dt)
    for g, r in zip(xa.download(), xb.download()):
        assert np.array_equal(g, r)
    a.set_diffusion(None)
    a.destroy()
    b.destroy()
    # per-member time steps: member 1 with its own dt, member 2 frozen
    m, opm = ah_domain(N, precision, members=3, order=42)
    m.set_diffusion(create_swm_diff_operator(diff_config(42), m))
    xm = create_stvec_swm(m)
    for k in range(3):
        xm.upload(*st, member=k)
    frozen = xm.download(member=2)
    create_timescheme(xm, "rk4").steps_members(xm, opm, [dt, 0.5 * dt, 0.0], 3)
    one, op1 = ah_domain(N, precision, order=42)
    d1 = create_swm_diff_operator(diff_config(42), one)
    x1 = create_stvec_swm(one).upload(*st)
    rk1, eul1 = create_timescheme(x1, "rk4"), create_timescheme(x1, "explicit_Eul1")
    for _ in range(3):
        rk1.step(x1, op1, one, 0.5 * dt)
        eul1.step(x1, d1, one, 0.5 * dt)
    tol = 1e-13 if precision == "fp64" else 1e-6
    for g, r in zip(xm.download(member=1), x1.download()):
        assert rel(g, r) < tol
    for g, r in zip(xm.download(member=2), frozen):
        assert np.array_equal(g, r)
    m.destroy()
    one.destroy()


def test_fp32_against_fp64_and_members():
    from ch_swe_b200 import create_stvec_swm, create_swm_diff_operator, create_timescheme
    from ch_swe_b200.testcases import williamson2
    N = 24
    base = williamson2(N, staggering="Ah")
    rng = np.random.default_rng(4)
    states = [tuple(f + 0.01 * np.abs(f).max() * rng.standard_normal(f.shape) for f in base) for _ in range(3)]
    out = {}
    for prec in ("fp64", "fp32"):
        dom, _ = ah_domain(N, prec, members=3)
        dif = create_swm_diff_operator(DIFF, dom)
        x = create_stvec_swm(dom)
        for m, s in enumerate(states):
            x.upload(*s, member=m)
        eul = create_timescheme(x, "explicit_Eul1")
        for _ in range(3):
            eul.step(x, dif, dom, 600.0)
        out[prec] = [x.download(member=m) for m in range(3)]
        dom.destroy()
    for m in range(3):
        for a, b in zip(out["fp32"][m], out["fp64"][m]):
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5
    # each member as a single-member context gives the same bits
    dom, _ = ah_domain(N, "fp64")
    dif = create_swm_diff_operator(DIFF, dom)
    x = create_stvec_swm(dom).upload(*states[1])
    eul = create_timescheme(x, "explicit_Eul1")
    for _ in range(3):
        eul.step(x, dif, dom, 600.0)
    for a, b in zip(x.download(), out["fp64"][1]):
        assert np.array_equal(a, b)
    dom.destroy()


def test_refusals():
    from ch_swe_b200 import SweError, create_domain, create_stvec_swm, create_swm_diff_operator, load
    ch = create_domain(16, precision="fp64")
    with pytest.raises(ValueError):
        create_swm_diff_operator(DIFF, ch)
    x, y = create_stvec_swm(ch), create_stvec_swm(ch)
    assert load().swe_diffusion_apply(ch.ctx, y.handle, x.handle, 21, 0.03, 0.01) != 0
    ch.destroy()
    dom, _ = ah_domain(16)
    with pytest.raises(ValueError):   # one order for both operators
        create_swm_diff_operator({**DIFF, "hordiff_h_name": "hordiff_scalar_Ah_sbp_42_narrow"}, dom)
    with pytest.raises(ValueError):
        create_swm_diff_operator(diff_config(43), dom)
    with pytest.raises(ValueError):   # the 6-3 closure blocks overlap below N = 17
        create_swm_diff_operator(diff_config(63), dom)
    x = create_stvec_swm(dom)
    assert load().swe_diffusion_step(dom.ctx, x.handle, 1.0, 43, 0.03, 0.01) != 0
    assert load().swe_diffusion_step(dom.ctx, x.handle, 1.0, 63, 0.03, 0.01) != 0
    dom.destroy()
    small, _ = ah_domain(8)
    with pytest.raises(ValueError):   # the 4-2 closure blocks overlap below N = 11
        create_swm_diff_operator(diff_config(42), small)
    x = create_stvec_swm(small)
    assert load().swe_diffusion_step(small.ctx, x.handle, 1.0, 42, 0.03, 0.01) != 0
    assert SweError is not None
    small.destroy()
