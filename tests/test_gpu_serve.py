"""Served mixed workload (continuous batching): every result equals the same
request run alone, the HBM budget bounds the pools, latencies are reported."""
import numpy as np
import pytest

from tests.conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu(lib_built):
    if not gpu_available():
        pytest.fail("no CUDA device: the -m gpu tests need a B200")


def _stream(n, seed, sizes=(24, 48), steps=(24, 64)):
    from ch_swe_b200.serve import poisson_stream
    return poisson_stream(n, rate=2000.0, seed=seed, sizes=sizes, steps=steps)


@pytest.mark.parametrize("grouped", [False, True])
def test_mixed_results_equal_alone_bitwise(grouped):
    """Same kernel configuration alone and in the mix: bit-identical states (both
    precisions, both operators); grouped: the linear pools of a precision tick as one
    group launch over their cube sizes."""
    from ch_swe_b200.serve import Server, run_alone
    reqs = _stream(20, 11, sizes=(24, 32, 48))
    srv = Server(hbm_budget_bytes=2 << 30, max_tick=8, max_slots={24: 6, 32: 4, 48: 4}, grouped=grouped)
    stats = srv.run(reqs, realtime=False)
    srv.close()
    assert stats.n == len(reqs)
    assert {r.operator for r in reqs} == {"linear", "advective"}
    assert (srv.group_ticks > 0) == grouped
    for r in reqs:
        alone = run_alone(r, kernel_config=r.pool_cfg)
        for a, b, name in zip(r.result, alone, "huv"):
            assert np.array_equal(a, b), (r.rid, r.N, r.precision, name, np.abs(a - b).max())


def test_mixed_fp64_matches_oracle():
    from ch_swe_b200.serve import Server
    from oracle.oracle import Oracle
    reqs = [r for r in _stream(16, 12, sizes=(24,), steps=(24, 40)) if r.precision == "fp64"][:4]
    assert {r.operator for r in reqs} == {"linear", "advective"}
    srv = Server(hbm_budget_bytes=1 << 30, max_tick=16)
    srv.run(reqs, realtime=False)
    srv.close()
    for r in reqs:
        o = Oracle(r.N, h_mean=r.h_mean, operator=r.operator)
        ref = o.rk4(*r.initial_state(), r.dt, r.nsteps)
        for a, b, name in zip(r.result, ref, "huv"):
            # 1e-12 of the field's scale; a wind that starts at rest is measured against
            # the gravity-wave speed sqrt(g H) (rounding in the gradient of the full
            # depth h ~ H is what separates the two FP64 results)
            scale = np.abs(b).max()
            if name != "h":
                scale = max(scale, np.sqrt(9.80616 * r.h_mean))
            assert np.abs(a - b).max() / scale < 1e-12, (r.rid, r.operator, name)


def test_budget_bounds_pools_and_all_requests_finish():
    from ch_swe_b200.serve import Server, member_bytes
    reqs = _stream(16, 13, sizes=(24, 48))
    budget = 3 * member_bytes(48, "fp64", "advective") + 2 * member_bytes(24, "fp64", "advective")
    srv = Server(hbm_budget_bytes=budget, max_tick=8)
    stats = srv.run(reqs, realtime=False)
    srv.close()
    assert stats.n == len(reqs)
    assert stats.peak_bytes <= budget
    assert all(r.result is not None for r in reqs)


def test_realtime_latencies_reported():
    from ch_swe_b200.serve import Server
    reqs = _stream(10, 14)
    srv = Server(hbm_budget_bytes=1 << 30, max_tick=16)
    stats = srv.run(reqs, realtime=True)
    srv.close()
    assert stats.n == 10
    assert all(r.latency > 0 for r in reqs)
    assert stats.p99_ms >= stats.p50_ms > 0
    assert stats.cell_updates_per_s > 0
