"""Group launches: the RK4 steps of several domains (mixed cube sizes and member
counts) as one grid per kernel give every domain the bits of its own steps with the
same kernel configuration; frozen members stay put; the launch count does not grow
with the number of domains; mismatched domains are refused."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


LINEAR = {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}


def _ics(N, M, seed):
    from ch_swe_b200.testcases import gaussian_hill
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(M):
        h, u, v = gaussian_hill(N, lam0=rng.uniform(0, 2 * np.pi), phi0=rng.uniform(-1.2, 1.2), d0=0.2,
                                amp=rng.uniform(0.5, 2.0))
        u = u + 0.1 * rng.standard_normal(u.shape)   # a wind that is not at rest
        out.append((h, u, v))
    return out


def _setup(sizes, precision, cfg, seed):
    """Domains of the given (N, members), their states with seeded ICs, H per member."""
    from ch_swe_b200 import create_domain, create_stvec_swm, create_swm_operator
    doms, states, ops, dts = [], [], [], []
    for k, (N, M) in enumerate(sizes):
        d = create_domain(N, precision=precision, n_members=M)
        d.kernel_config = cfg
        op = create_swm_operator(d.grav, LINEAR, d)
        st = create_stvec_swm(d)
        for m, ic in enumerate(_ics(N, M, seed + k)):
            st.upload(*ic, member=m)
            op.set_member_h_mean(m, 800.0 + 100.0 * m + 37.0 * k)
        doms.append(d)
        states.append(st)
        ops.append(op)
        dts.append(np.array([3600.0 / N * (1 + 0.1 * m) for m in range(M)]))
    return doms, states, ops, dts


@pytest.mark.parametrize("precision,cfg", [("fp32", (25, 3, 0)), ("fp64", (17, 4, 0)), ("fp32", (33, 2, 0))])
def test_group_bitwise_equals_alone(precision, cfg):
    from ch_swe_b200 import create_timescheme
    from ch_swe_b200.swm import create_group
    sizes = [(24, 3), (48, 2), (96, 1), (32, 2)]
    nsteps = 11   # one graph of eight steps and three single steps
    gd, gs, _, dts = _setup(sizes, precision, cfg, 100)
    ad, ast, aops, _ = _setup(sizes, precision, cfg, 100)
    dts[1][1] = 0.0   # a frozen member
    frozen = gs[1].download(member=1)
    grp = create_group(gd)
    grp.steps_members(gs, dts, nsteps)
    grp.synchronize()
    assert grp.launches == 12 * nsteps
    for k, (N, M) in enumerate(sizes):
        rk = create_timescheme(ast[k], "rk4")
        rk.steps_members(ast[k], aops[k], dts[k], nsteps)
        ad[k].synchronize()
        for m in range(M):
            for a, b, name in zip(gs[k].download(member=m), ast[k].download(member=m), "huv"):
                assert np.array_equal(a, b), (N, m, name, np.abs(a - b).max())
    for a, b in zip(gs[1].download(member=1), frozen):
        assert np.array_equal(a, b)
    grp.destroy()
    for d in gd + ad:
        d.destroy()


def test_group_refuses_mismatched_domains():
    from ch_swe_b200 import SweError, create_domain
    from ch_swe_b200.swm import create_group
    a = create_domain(24, precision="fp32")
    b = create_domain(32, precision="fp64")
    c = create_domain(24, precision="fp32")
    d = create_domain(24, precision="fp32", operator="advective")
    for x in (a, b, c):
        x.kernel_config = (25, 3, 0)
    c.kernel_config = (17, 4, 0)
    for pair in ((a, b), (a, c), (a, d), (a, a)):
        with pytest.raises(SweError):
            create_group(list(pair))
    a.kernel_config = (25, 2, 0)   # a split configuration without a group launch
    with pytest.raises(SweError):
        create_group([a])
    for x in (a, b, c, d):
        x.destroy()
