"""GPU diagnostics (swe_diag through the C ABI) against the oracle's restatement of
swm_output_diag_t's CFL and extrema."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built, oracle_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_diag_matches_oracle(precision, tol):
    from ch_swe_b200 import create_domain, create_stvec_swm
    from ch_swe_b200.diag import SwmOutputDiag
    from oracle.oracle import Oracle
    N, dt = 24, 450.0
    o = Oracle(N, h_mean=1000.0)
    h = o.gaussian(lam0=0.4, phi0=0.3, d0=0.3, amp=5.0)[0] - 1.0
    _, u, v = o.ts2(u0=30.0, h_mean=1000.0, axis=(0.3, 0.0, 0.95), linear_mode=True)
    ref = o.diag(h, u, v, dt)
    dom = create_domain(N, precision=precision, h_mean=1000.0, n_members=2)
    st = create_stvec_swm(dom)
    st.upload(h, u, v, member=1)
    st.upload(h * 0, u * 0, v * 0, member=0)
    d = SwmOutputDiag(dom).diagnostics(st, dt, member=1)
    got = (d["h_min"], d["h_max"], d["cfl_gravity"], d["cfl_adv_x"], d["cfl_adv_y"])
    for g, r, name in zip(got, ref, ("h_min", "h_max", "cfl_gravity", "cfl_adv_x", "cfl_adv_y")):
        assert abs(g - r) <= tol * max(abs(r), 1e-30), (name, g, r)
    d0 = SwmOutputDiag(dom).diagnostics(st, dt, member=0)
    assert d0["h_max"] == 0.0 and d0["cfl_adv_x"] == 0.0
    dom.destroy()
