"""Served mixed workload: continuous batching of shallow-water integrations on one GPU.

A request is one integration: operator (linear or advective), cube size N,
precision, number of RK4 steps, time step, depth and an initial state (h, u, v).
The server keeps one *pool* per (operator, N, precision): a context with a fixed
number of member slots, its own CUDA stream and its states resident in HBM.  A request occupies one slot from
admission to completion.

Continuous batching:
- every pool advances all of its occupied slots together in *ticks* of at most
  `max_tick` RK4 steps (one graph replay per step, `swe_rk4_steps_members`);
  free slots have time step 0 and cost nothing (their blocks exit at once);
- a tick is as long as the shortest remaining integration in the pool, so every
  request stops exactly at its own step count;
- between ticks, finished requests leave (their state is downloaded) and queued
  requests of that pool are uploaded into the free slots;
- pools run on separate streams, so the work of different cube sizes and
  precisions overlaps on the device;
- with grouped=True, the linear pools of one precision up to cube size
  group_max_n share one kernel configuration and tick together as a group
  (swe_group_rk4_steps_members): one grid per kernel covers every cube size of the
  group, twelve launches per RK4 step for all of them; the tick is as long as the
  shortest remaining integration of the group.  Larger cubes fill the GPU with one
  member and keep their own pools, streams and autotuned configurations.

Admission by HBM budget: a pool is created when a request needs one and its
slots fit in the budget that other pools leave free (idle empty pools are
released to make room); requests wait in the queue until a slot frees up.

The reference has no server: it integrates one state per run
(src/models/shallow_water/shallow_water_mod.f90:112-143).  Each served result
is the same as the same request run alone (tests/test_gpu_serve.py).
"""
from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field

import numpy as np

from . import ensemble, testcases

SIZES = (24, 48, 96, 192, 384)
MAX_SLOTS = {24: 64, 48: 64, 96: 32, 192: 16, 384: 8}


def stable_dt(N: int) -> float:
    """RK4 time step of the served linear runs: 150 s at C192, scaled with the grid spacing."""
    return 150.0 * 192.0 / N


def member_bytes(N: int, precision: str, operator: str = "linear") -> int:
    """Device bytes one member slot of a pool holds: the state, two stage buffers,
    the RK accumulator, the contravariant scratch, the FP32 compensation, the edge
    buffer and the edge strips (layout of swe_api.cu); the advective operator adds
    the mass flux, the advective tendencies, uh/vh, the flux strips, the virtual
    wind points and the boundary h."""
    elem = 4 if precision == "fp32" else 8
    rows = N + 9
    pitch = (rows + 7) // 8 * 8
    box = 3 * 6 * rows * pitch
    words = 5 * box + 6 * 4 * (N + 1) * (3 + 4)
    if operator == "advective":
        words += 3 * box + 6 * 4 * (N + 1) * (4 + 1) + 6 * (24 * N + 12)
    extra = box * 4 if precision == "fp32" else 0
    return words * elem + extra


@dataclass
class Request:
    rid: int
    N: int
    precision: str
    nsteps: int
    dt: float
    h_mean: float
    ic_params: tuple            # (centres, widths, amps) of the Gaussian bumps, or (h, u, v) arrays
    arrival: float = 0.0
    operator: str = "linear"
    # filled by the server
    admitted: float | None = None
    finished: float | None = None
    pool_tile: int | None = None
    pool_cfg: tuple | None = None
    result: tuple | None = None

    _ic: tuple | None = None

    @property
    def ic(self):
        """Initial (h, u, v), FP64 host arrays (generated on first use)."""
        if self._ic is None:
            p = self.ic_params
            if len(p) == 3 and isinstance(p[0], np.ndarray):
                self._ic = p
            else:
                self._ic = testcases.gaussian_sum(self.N, *p)
        return self._ic

    def initial_state(self):
        """(h, u, v) as uploaded: the linear operator integrates the perturbation of
        the mean depth h_mean, the advective one the full depth h_mean + bumps."""
        h, u, v = self.ic
        return (h + self.h_mean, u, v) if self.operator == "advective" else (h, u, v)

    @property
    def cell_updates(self) -> int:
        return 6 * self.N * self.N * self.nsteps

    @property
    def latency(self) -> float | None:
        return None if self.finished is None else self.finished - self.arrival


def poisson_stream(n_requests: int, rate: float = 200.0, seed: int = 20261203 + 5, sizes=SIZES,
                   steps=(24, 576), precisions=("fp32", "fp64"), operators=("linear", "advective")):
    """Seeded Poisson arrivals (mean `rate` per second); N uniform over `sizes`, steps
    uniform in `steps`, precision and operator 50/50; each request one ensemble-style
    initial state (H ~ U[500, 2000] m, 1-4 Gaussians, at rest)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for k in range(n_requests):
        t += rng.exponential(1.0 / rate)
        N = int(rng.choice(sizes))
        nst = int(rng.integers(steps[0], steps[1] + 1))
        prec = str(rng.choice(precisions))
        op = str(rng.choice(operators))
        H, centres, widths, amps = ensemble.member_params(1, int(rng.integers(1 << 31)))[0]
        reqs.append(Request(k, N, prec, nst, stable_dt(N), H, (centres, widths, amps), arrival=t, operator=op))
    return reqs


def _operator(dom, operator: str):
    from .swm import create_swm_operator
    if operator == "advective":
        return create_swm_operator(dom.grav, {"swm_operator_type": "advective_swm_operator"}, dom)
    return create_swm_operator(dom.grav, {"swm_operator_type": "linear_swm_operator", "h_mean": 1000.0}, dom)


# Kernel configuration of grouped pools (a configuration with a group launch).
GROUP_CONFIG = {"fp32": (25, 3, 0), "fp64": (25, 3, 0)}


class Pool:
    """Member slots of one (operator, N, precision): one context on its own stream.
    kernel_config: a fixed (tile, blocks per SM, runs) instead of the tile or the
    autotuner's choice."""

    def __init__(self, N: int, precision: str, capacity: int, torch, tile=None, operator: str = "linear",
                 kernel_config=None):
        from .swm import create_domain, create_stvec_swm, create_timescheme
        self.N, self.precision, self.capacity, self.operator = N, precision, capacity, operator
        self.torch = torch
        self.stream = torch.cuda.Stream()
        self.dom = create_domain(N, precision=precision, n_members=capacity, operator=operator)
        self.dom.set_stream(self.stream.cuda_stream)
        self.grouped = kernel_config is not None
        if kernel_config is not None:
            self.dom.kernel_config = kernel_config
        elif tile is None:
            with torch.cuda.stream(self.stream):
                self.dom.autotune(nreps=4)
        else:
            self.dom.tile = tile
        self.op = _operator(self.dom, operator)
        self.state = create_stvec_swm(self.dom)
        self.rk = create_timescheme(self.state, "rk4")
        self.slots: list[Request | None] = [None] * capacity
        self.remaining = [0] * capacity
        self.event = None
        self.tick_len = 0
        self.bytes = capacity * member_bytes(N, precision, operator)

    @property
    def busy(self) -> bool:
        return self.event is not None

    @property
    def occupied(self) -> int:
        return sum(r is not None for r in self.slots)

    def free_slot(self):
        for k, r in enumerate(self.slots):
            if r is None:
                return k
        return None

    def admit(self, req: Request, now: float):
        k = self.free_slot()
        self.state.upload(*req.initial_state(), member=k)
        if req.operator == "linear":
            self.op.set_member_h_mean(k, req.h_mean)
        self.slots[k] = req
        self.remaining[k] = req.nsteps
        req.admitted = now
        req.pool_tile = self.dom.tile
        req.pool_cfg = self.dom.kernel_config

    def active(self):
        return [k for k, r in enumerate(self.slots) if r is not None and self.remaining[k] > 0]

    def tick_dts(self):
        """Per-slot time steps of the next tick (0: a free or finished slot)."""
        dts = np.zeros(self.capacity)
        for k in self.active():
            dts[k] = self.slots[k].dt
        return dts

    def launch_tick(self, max_tick: int):
        active = self.active()
        if not active:
            return False
        L = min(max_tick, min(self.remaining[k] for k in active))
        dts = self.tick_dts()
        with self.torch.cuda.stream(self.stream):
            self.rk.steps_members(self.state, self.op, dts, L)
            self.event = self.torch.cuda.Event()
            self.event.record(self.stream)
        self.tick_len = L
        return True

    def poll(self, now_fn):
        """If the tick in flight has finished: account it, retire finished requests."""
        if self.event is None or not self.event.query():
            return []
        self.event = None
        done = []
        for k, r in enumerate(self.slots):
            if r is None or self.remaining[k] <= 0:
                continue
            self.remaining[k] -= self.tick_len
            if self.remaining[k] == 0:
                r.result = self.state.download(member=k)
                r.finished = now_fn()
                self.slots[k] = None
                done.append(r)
        return done

    def destroy(self):
        self.dom.destroy()


@dataclass
class ServeStats:
    n: int
    makespan_s: float
    p50_ms: float
    p99_ms: float
    mean_ms: float
    requests_per_s: float
    cell_updates_per_s: float
    pools: dict = field(default_factory=dict)
    peak_bytes: int = 0
    # service time (admission to finish) and queue wait (arrival to admission)
    service_p50_ms: float = 0.0
    service_p99_ms: float = 0.0
    wait_p50_ms: float = 0.0
    wait_p99_ms: float = 0.0


class Server:
    def __init__(self, hbm_budget_bytes: int = 16 << 30, max_tick: int = 16, max_slots=None, tiles=None,
                 grouped: bool = False, group_max_n: int = 96):
        import torch
        self.torch = torch
        self.budget = int(hbm_budget_bytes)
        self.max_tick = int(max_tick)
        self.max_slots = dict(MAX_SLOTS if max_slots is None else max_slots)
        self.tiles = dict(tiles or {})
        self.grouped = bool(grouped)
        self.group_max_n = int(group_max_n)
        self.pools: dict[tuple, Pool] = {}
        # precision -> (the grouped pools' keys, DomainGroup)
        self.groups: dict[str, tuple] = {}
        self.peak = 0
        self.group_ticks = 0

    def used_bytes(self) -> int:
        return sum(p.bytes for p in self.pools.values())

    def pool_capacity(self, key) -> int:
        """Slots a pool of key (N, precision, operator) gets when the budget is free."""
        N, precision, operator = key
        return int(min(self.max_slots.get(N, 4), self.budget // member_bytes(N, precision, operator)))

    def pretune(self, keys, nreps: int = 16):
        """Autotune the stage kernels of the pools of `keys` one after another on an idle
        device, before requests arrive.  The choices go to the library's process-wide
        tuning cache, so pools created while serving take them instead of timing
        under the load of the other pools."""
        from .swm import create_domain
        for key in sorted(set(keys)):
            if key in self.tiles:
                continue
            N, precision, operator = key
            cap = self.pool_capacity(key)
            if cap < 1:
                continue
            dom = create_domain(N, precision=precision, n_members=cap, operator=operator)
            dom.autotune(nreps=nreps)
            dom.destroy()

    def _pool_for(self, req: Request):
        if req.operator not in ("linear", "advective"):
            raise ValueError(f"request {req.rid}: operator {req.operator!r} is not served")
        key = (req.N, req.precision, req.operator)
        if key in self.pools:
            return self.pools[key]
        per = member_bytes(req.N, req.precision, req.operator)
        want = self.max_slots.get(req.N, 4)
        free = self.budget - self.used_bytes()
        if free < per:
            # release idle, empty pools of other keys (and the groups that hold them)
            for k2, p in list(self.pools.items()):
                if not p.busy and p.occupied == 0 and not self._group_busy(k2):
                    self._drop_group(k2[1])
                    p.destroy()
                    del self.pools[k2]
            free = self.budget - self.used_bytes()
        cap = min(want, free // per)
        if cap < 1:
            return None
        cfg = (GROUP_CONFIG[req.precision]
               if self.grouped and req.operator == "linear" and req.N <= self.group_max_n else None)
        pool = Pool(req.N, req.precision, int(cap), self.torch, tile=self.tiles.get(key), operator=req.operator,
                    kernel_config=cfg)
        self.pools[key] = pool
        self.peak = max(self.peak, self.used_bytes())
        return pool

    def _grouped_pools(self, precision: str):
        return sorted((k for k, p in self.pools.items() if p.grouped and k[1] == precision), key=lambda k: k[0])

    def _group_busy(self, key) -> bool:
        return any(self.pools[k].busy for k in self._grouped_pools(key[1])) if self.pools[key].grouped else False

    def _drop_group(self, precision: str):
        g = self.groups.pop(precision, None)
        if g is not None:
            g[1].destroy()

    def _group_tick(self, precision: str) -> bool:
        """One tick of every grouped pool of `precision` as one group launch (all of
        them idle)."""
        from .swm import create_group
        keys = self._grouped_pools(precision)
        pools = [self.pools[k] for k in keys]
        if not pools or any(p.busy for p in pools):
            return False
        active = [(p, k) for p in pools for k in p.active()]
        if not active:
            return False
        L = min(self.max_tick, min(p.remaining[k] for p, k in active))
        g = self.groups.get(precision)
        if g is None or g[0] != keys:
            self._drop_group(precision)
            g = (keys, create_group([p.dom for p in pools]))
            self.groups[precision] = g
        g[1].steps_members([p.state for p in pools], [p.tick_dts() for p in pools], L)
        ev = self.torch.cuda.Event()
        ev.record(pools[0].stream)
        for p in pools:
            p.event = ev
            p.tick_len = L
        self.group_ticks += 1
        return True

    def run(self, requests, realtime: bool = True) -> ServeStats:
        """Serve `requests` (arrival times in seconds from the start); realtime=False
        admits every request at once in arrival order (for tests)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        queue: collections.deque[Request] = collections.deque()
        t0 = time.perf_counter()
        now = (lambda: time.perf_counter() - t0) if realtime else (lambda: 0.0)
        if not realtime:
            for r in pending:
                r.arrival = 0.0
        done = []
        total = len(pending)
        while len(done) < total:
            progressed = False
            t = now()
            while pending and pending[0].arrival <= t:
                queue.append(pending.popleft())
                progressed = True
            for p in list(self.pools.values()):
                fin = p.poll(now)
                if fin:
                    done.extend(fin)
                    progressed = True
            # admission into free slots of idle pools, in arrival order
            waiting = collections.deque()
            while queue:
                r = queue.popleft()
                p = self._pool_for(r)
                if p is not None and not p.busy and p.free_slot() is not None:
                    p.admit(r, now())
                    progressed = True
                else:
                    waiting.append(r)
            queue = waiting
            for p in self.pools.values():
                if not p.grouped and not p.busy and p.launch_tick(self.max_tick):
                    progressed = True
            for prec in ("fp32", "fp64"):
                if self._group_tick(prec):
                    progressed = True
            if not progressed:
                time.sleep(20e-6)
        makespan = max(r.finished for r in done) - min(r.arrival for r in done) if realtime else time.perf_counter() - t0
        lat = np.array([r.latency for r in done]) * 1e3 if realtime else np.array([0.0])
        svc = np.array([r.finished - r.admitted for r in done]) * 1e3 if realtime else np.array([0.0])
        wait = np.array([r.admitted - r.arrival for r in done]) * 1e3 if realtime else np.array([0.0])
        cells = sum(r.cell_updates for r in done)
        return ServeStats(
            n=len(done), makespan_s=makespan, p50_ms=float(np.percentile(lat, 50)),
            p99_ms=float(np.percentile(lat, 99)), mean_ms=float(lat.mean()),
            requests_per_s=len(done) / makespan, cell_updates_per_s=cells / makespan,
            pools={f"{k[2]}/C{k[0]}/{k[1]}": {"slots": p.capacity, "kernel_config": list(p.dom.kernel_config),
                                              "grouped": p.grouped} for k, p in self.pools.items()},
            peak_bytes=self.peak,
            service_p50_ms=float(np.percentile(svc, 50)), service_p99_ms=float(np.percentile(svc, 99)),
            wait_p50_ms=float(np.percentile(wait, 50)), wait_p99_ms=float(np.percentile(wait, 99)))

    def close(self):
        for prec in list(self.groups):
            self._drop_group(prec)
        for p in self.pools.values():
            p.destroy()
        self.pools.clear()


def run_alone(req: Request, tile=None, kernel_config=None):
    """The same integration in its own single-member context (the comparison arm)."""
    from .swm import create_domain, create_stvec_swm, create_timescheme
    dom = create_domain(req.N, precision=req.precision, operator=req.operator)
    if kernel_config is not None:
        dom.kernel_config = kernel_config
    elif tile is not None:
        dom.tile = tile
    op = _operator(dom, req.operator)
    if req.operator == "linear":
        op.set_member_h_mean(0, req.h_mean)
    st = create_stvec_swm(dom).upload(*req.initial_state())
    create_timescheme(st, "rk4").steps_members(st, op, [req.dt], req.nsteps)
    out = st.download()
    dom.destroy()
    return out
