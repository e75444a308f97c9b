"""Host-side pieces of the serving loop (no GPU): the seeded request stream and
the per-slot memory model."""
import numpy as np


def test_poisson_stream_is_seeded_and_in_range():
    from ch_swe_b200.serve import poisson_stream, SIZES
    a = poisson_stream(200, rate=200.0, seed=5)
    b = poisson_stream(200, rate=200.0, seed=5)
    assert [(r.N, r.nsteps, r.precision, r.arrival) for r in a] == [(r.N, r.nsteps, r.precision, r.arrival) for r in b]
    assert all(r.N in SIZES and 24 <= r.nsteps <= 576 and r.precision in ("fp32", "fp64") for r in a)
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    rate = len(arr) / arr[-1]
    assert 150 < rate < 260
    assert 0.35 < np.mean([r.precision == "fp32" for r in a]) < 0.65
    assert 0.35 < np.mean([r.operator == "advective" for r in a]) < 0.65
    h, u, v = a[0].ic
    assert h.shape == (6, a[0].N + 1, a[0].N + 1) and not u.any() and not v.any()


def test_member_bytes_and_dt():
    from ch_swe_b200.serve import member_bytes, stable_dt
    assert member_bytes(48, "fp64") > member_bytes(48, "fp32") > member_bytes(24, "fp32")
    assert member_bytes(48, "fp32", "advective") > member_bytes(48, "fp32", "linear")
    # five FP64 boxes of 3 fields x 6 panels x (N+9) x pitch dominate
    N = 192
    rows = N + 9
    pitch = (rows + 7) // 8 * 8
    assert member_bytes(N, "fp64") >= 5 * 18 * rows * pitch * 8
    assert stable_dt(192) == 150.0 and stable_dt(384) == 75.0


def test_pool_capacity_follows_budget():
    """A pool gets its size's slot count while the budget allows, fewer when it does
    not, and none when one member does not fit (the capacity pretune tunes for)."""
    from ch_swe_b200.serve import MAX_SLOTS, Server, member_bytes
    per = member_bytes(192, "fp64", "advective")
    big = Server(hbm_budget_bytes=64 << 30)
    assert big.pool_capacity((192, "fp64", "advective")) == MAX_SLOTS.get(192, 4)
    small = Server(hbm_budget_bytes=2 * per + 1)
    assert small.pool_capacity((192, "fp64", "advective")) == min(MAX_SLOTS.get(192, 4), 2)
    assert Server(hbm_budget_bytes=per - 1).pool_capacity((192, "fp64", "advective")) == 0
