"""The C-grid operators on the GPU (swe_c_grad, swe_c_div and swe_operator_contravariant
on a C-staggered context) against the CPU FP64 oracle: within 1e-12 relative (max norm)
in FP64 and 1e-5 in FP32, on random fields, at sizes with one and several thread blocks
per panel.  A C context rejects the linear operator, as the reference aborts in its
C-grid Coriolis operator."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built, oracle_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


def rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("N", [8, 16, 31, 40, 65])
def test_c_operators_match_oracle(N, precision):
    from ch_swe_b200 import create_domain, create_stvec_swm, state_shapes
    from ch_swe_b200.swm import create_co2contra_operator, create_div_operator, create_grad_operator
    from oracle.oracle import Oracle
    rng = np.random.default_rng(900 + N)
    h, u, v = (rng.standard_normal(s) for s in state_shapes(N, staggering="C"))
    o = Oracle(N)
    ref_g = o.c_grad(h)
    ref_d = o.c_div(u, v)
    ref_c = o.c_co2contra(u, v)
    dom = create_domain(N, precision=precision, horizontal_staggering="C")
    x = create_stvec_swm(dom).upload(h, u, v)
    y = create_stvec_swm(dom).upload(h, u, v)
    tol = 1e-12 if precision == "fp64" else 1e-5
    create_grad_operator(dom, "grad_c_sbp_sat_42").calc_grad(y, x)
    _, gx, gy = y.download()
    assert rel(gx, ref_g[0]) < tol and rel(gy, ref_g[1]) < tol, (rel(gx, ref_g[0]), rel(gy, ref_g[1]))
    create_div_operator(dom, "div_c_sbp_sat_42").calc_div(y, x)
    d, _, _ = y.download()
    assert rel(d, ref_d) < tol, rel(d, ref_d)
    create_co2contra_operator(dom, "co2contra_c_sbp42_new").transform(y, x)
    _, ut, vt = y.download()
    assert rel(ut, ref_c[0]) < tol and rel(vt, ref_c[1]) < tol, (rel(ut, ref_c[0]), rel(vt, ref_c[1]))
    dom.destroy()


def test_c_operators_members_independent():
    from ch_swe_b200 import create_domain, create_stvec_swm, state_shapes
    from ch_swe_b200.swm import create_div_operator, create_grad_operator
    from oracle.oracle import Oracle
    N, M = 20, 3
    rng = np.random.default_rng(11)
    states = [tuple(rng.standard_normal(s) for s in state_shapes(N, staggering="C")) for _ in range(M)]
    dom = create_domain(N, n_members=M, horizontal_staggering="C")
    x, y = create_stvec_swm(dom), create_stvec_swm(dom)
    for k in range(M):
        x.upload(*states[k], member=k)
        y.upload(*states[k], member=k)
    create_grad_operator(dom, "grad_c_sbp_sat_42").calc_grad(y, x)
    o = Oracle(N)
    for k in range(M):
        _, gx, gy = y.download(member=k)
        ref = o.c_grad(states[k][0])
        assert rel(gx, ref[0]) < 1e-12 and rel(gy, ref[1]) < 1e-12
    create_div_operator(dom, "div_c_sbp_sat_42").calc_div(y, x)
    for k in range(M):
        d, _, _ = y.download(member=k)
        assert rel(d, o.c_div(states[k][1], states[k][2])) < 1e-12
    dom.destroy()


def test_c_context_rejects_the_linear_operator():
    from ch_swe_b200 import SweError, create_domain, create_stvec_swm, create_swm_operator, create_timescheme
    dom = create_domain(12, horizontal_staggering="C")
    op = create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)
    x, y = create_stvec_swm(dom), create_stvec_swm(dom)
    with pytest.raises(SweError, match="calc_coriolis"):
        op.apply(y, x, dom)
    with pytest.raises(SweError, match="calc_coriolis"):
        create_timescheme(x, "rk4").steps(x, op, dom, 60.0, 2)
    dom.destroy()
