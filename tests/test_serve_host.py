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


def test_group_tick_host_logic(monkeypatch):
    """Grouped pools of one precision tick together: one group call per tick, the tick
    as long as the shortest remaining integration of the group, time step 0 for free
    slots, one shared completion event, and a new group when a pool joins."""
    import ch_swe_b200.swm as swm
    from ch_swe_b200.serve import Request, Server

    calls, made = [], []

    class FakeGroup:
        def __init__(self, doms):
            self.doms = doms
            made.append(self)

        def steps_members(self, states, dts, n):
            calls.append((self, list(states), [np.array(x) for x in dts], n))

        def destroy(self):
            pass

    class FakeEvent:
        def record(self, stream):
            self.stream = stream

        def query(self):
            return True

    class FakeTorch:
        class cuda:
            Event = FakeEvent

    class FakePool:
        def __init__(self, N, cap):
            self.N, self.capacity, self.grouped, self.operator, self.precision = N, cap, True, "linear", "fp32"
            self.slots, self.remaining = [None] * cap, [0] * cap
            self.dom, self.state, self.stream = f"dom{N}", f"st{N}", f"stream{N}"
            self.event, self.tick_len = None, 0

        busy = property(lambda self: self.event is not None)

        def active(self):
            return [k for k, r in enumerate(self.slots) if r is not None and self.remaining[k] > 0]

        def tick_dts(self):
            d = np.zeros(self.capacity)
            for k in self.active():
                d[k] = self.slots[k].dt
            return d

    monkeypatch.setattr(swm, "create_group", FakeGroup)
    srv = Server.__new__(Server)
    srv.torch, srv.max_tick, srv.pools, srv.groups, srv.group_ticks = FakeTorch, 16, {}, {}, 0
    a, b = FakePool(48, 3), FakePool(24, 2)
    srv.pools = {(48, "fp32", "linear"): a, (24, "fp32", "linear"): b}
    a.slots[1], a.remaining[1] = Request(0, 48, "fp32", 40, 300.0, 1000.0, None), 40
    b.slots[0], b.remaining[0] = Request(1, 24, "fp32", 9, 600.0, 1000.0, None), 9
    assert srv._group_tick("fp32") and not srv._group_tick("fp64")
    g, states, dts, n = calls[-1]
    assert n == 9 and states == ["st24", "st48"] and g.doms == ["dom24", "dom48"]
    assert dts[0].tolist() == [600.0, 0.0] and dts[1].tolist() == [0.0, 300.0, 0.0]
    assert a.event is b.event and a.tick_len == b.tick_len == 9
    assert not srv._group_tick("fp32")          # busy until polled
    a.event = b.event = None
    b.remaining[0] = 0
    assert srv._group_tick("fp32") and calls[-1][3] == 16 and len(made) == 1
    a.event = b.event = None
    c = FakePool(96, 1)
    srv.pools[(96, "fp32", "linear")] = c
    assert srv._group_tick("fp32") and len(made) == 2 and made[-1].doms == ["dom24", "dom48", "dom96"]
