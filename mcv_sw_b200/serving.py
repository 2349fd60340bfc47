"""Forecast serving on one B200: continuous batching over the C ABI.

Forecast requests of different order, Nc and length arrive over time.  The
server groups them by grid (order, Nc): each group owns one or more pools, a
pool being one handle with `slots` device-resident member slots.  A request is
admitted into a free slot of an idle pool of its group, or into a new pool
when the HBM budget has room for that pool's footprint
(mcv_footprint_bytes); otherwise it waits.  Every idle pool with active
members is advanced by a chunk of steps on its own stream (mcv_set_active
selects the slots, mcv_step_async queues the chunk), so pools of different
groups run on the GPU at the same time; finished chunks are found with
mcv_query, finished forecasts are checked for non-finite values, downloaded
and their slots freed for the next requests.  A request's result does not
depend on what else runs: each member's arithmetic reads only that member's
data, whatever slot, pool or launch it shares.

With device_setup the pools build their geometry on the device
(mcv_set_geometry_equiangular) and a request that carries a seeded spec
instead of host arrays is admitted by generating its initial state on the
device (mcv_set_member_balanced_flow): nothing of the state crosses PCIe.

The reference runs one forecast per process (src/MCV_SW.F90); it has no
serving layer.  `run_one_at_a_time` is the plain loop the server is compared
with: one request after the other, each on its own single-member handle.
"""
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import api, cases


@dataclass
class Request:
    id: int
    arrival: float  # seconds after the stream starts
    order: int
    nc: int
    hours: float  # forecast length; rounded up to whole steps of the group's dt
    phi_s: np.ndarray = None  # initial state as host arrays, or ...
    u: np.ndarray = None
    v: np.ndarray = None
    phi: np.ndarray = None
    spec: dict = None  # ... a seeded balanced-flow spec generated on the device

    @property
    def key(self):
        return (self.order, self.nc)


@dataclass
class Result:
    id: int
    order: int
    nc: int
    nsteps: int
    dt: float
    arrival: float
    admitted: float
    finished: float
    finite: bool = True
    state: dict = field(default=None, repr=False)

    @property
    def latency(self):
        return self.finished - self.arrival

    @property
    def sim_days(self):
        return self.nsteps * self.dt / 86400.0


def make_requests(count, seed=4, rate=20.0, radius=cases.EARTH_RADIUS, geoms=None, specs=False):
    """The seeded serving stream: Poisson arrivals, MCV3/MCV4 with probability
    0.5, Nc from {48, 96, 192, 384} (0.4/0.3/0.2/0.1), 6-120 h, balanced tilted
    zonal flow + seeded harmonics, half with a seeded mountain.  specs=True:
    requests carry the seeded spec instead of host arrays (device admission)."""
    geoms = {} if geoms is None else geoms
    out = []
    for r in cases.serving_requests(seed=seed, rate=rate, count=count):
        if specs:
            out.append(Request(r["id"], r["t"], r["order"], r["nc"], r["hours"], spec=cases.serving_spec(radius, r)))
            continue
        key = (r["order"], r["nc"])
        if key not in geoms:
            geoms[key] = api.Geometry(r["order"], r["nc"], radius)
        st = cases.serving_state(geoms[key], r)
        out.append(Request(r["id"], r["t"], r["order"], r["nc"], r["hours"], st.phi_s, st.u, st.v, st.phi))
    return out, geoms


class _Pool:
    """One handle of a group: `slots` member slots on one (order, Nc) grid."""

    def __init__(self, server, key, slots):
        self.key, self.slots = key, slots
        self.dt = server.group_dt(key)
        self.bytes = server.footprint(key, slots)
        self.stepper = server.stepper_factory(key[0], key[1], self.dt, server.scheme, members=slots,
                                              precision=server.precision, radius=server.radius)
        if server.device_setup:
            self.stepper.set_geometry_equiangular()
        else:
            self.stepper.set_geometry(server.geometry(key))
        self.req = [None] * slots  # request held by each slot
        self.left = [0] * slots  # steps still to take
        self.admitted = [0.0] * slots
        self.active = []  # slots advanced by the next chunk
        self.device_active = None  # slot list the handle was last given
        self.in_flight = 0  # steps of the chunk on the GPU (0: idle)
        self.launched = 0.0
        self.ms_per_step = None

    def free_slot(self):
        for s in range(self.slots):
            if self.req[s] is None:
                return s
        return None

    def close(self):
        self.stepper.close()


class ForecastServer:
    """Continuous-batching request loop (see the module docstring).

    precision/scheme: arithmetic and RK scheme of every forecast (RK3_TVD, the
    cheaper scheme, by default).  hbm_budget: bytes the pools may hold (default
    85% of the device's free memory when the server starts).  slot_bytes: a
    pool gets as many slots as fit in this many bytes (1..max_slots).
    chunk_ms: target GPU time of one chunk, which bounds how long an arriving
    request waits for a busy pool.  tile: stage-kernel tile index used by every
    pool (None: each pool's autotuner chooses); split-precision results are
    reproducible bit for bit only on the same tile shape.  device_setup: pools
    build their geometry on the device, and requests carrying a spec get their
    initial state generated there."""

    def __init__(self, precision="mixed", scheme="RK3_TVD", hbm_budget=None, slot_bytes=8e9, max_slots=32,
                 chunk_ms=25.0, tile=None, radius=cases.EARTH_RADIUS, keep_states=False, poll_s=2e-4,
                 geoms=None, stepper_factory=None, footprint_fn=None, memory_fn=None, clock=time.perf_counter,
                 device_setup=False):
        self.precision, self.scheme, self.radius = precision, scheme, radius
        self.device_setup = device_setup
        self.slot_bytes, self.max_slots, self.chunk_ms = slot_bytes, max_slots, chunk_ms
        self.tile, self.keep_states, self.poll_s, self.clock = tile, keep_states, poll_s, clock
        self.stepper_factory = stepper_factory or api.Stepper
        self.footprint_fn = footprint_fn or api.footprint_bytes
        if hbm_budget is None:
            free, _ = (memory_fn or api.device_memory)()
            hbm_budget = int(0.85 * free)
        self.budget = int(hbm_budget)
        self.geoms = {} if geoms is None else geoms
        self.dts = {}
        self.pools = []
        self.stats = {"pools_created": 0, "pools_evicted": 0, "chunks": 0, "max_concurrent_pools": 0}

    # ---- per-group constants ----
    def geometry(self, key):
        if key not in self.geoms:
            self.geoms[key] = api.Geometry(key[0], key[1], self.radius)
        return self.geoms[key]

    def group_dt(self, key):
        if key not in self.dts:
            self.dts[key] = cases.serving_dt(self.geometry(key))
        return self.dts[key]

    def nsteps(self, req):
        return max(1, int(math.ceil(req.hours * 3600.0 / self.group_dt(req.key) - 1e-9)))

    def footprint(self, key, slots):
        return int(self.footprint_fn(key[0], key[1], self.scheme, self.precision, slots))

    def slots_for(self, key):
        per_member = self.footprint(key, 2) - self.footprint(key, 1)
        return max(1, min(self.max_slots, int(self.slot_bytes // max(per_member, 1))))

    @property
    def used(self):
        return sum(p.bytes for p in self.pools)

    # ---- pools ----
    def _new_pool(self, key):
        """A pool of slots_for(key) slots, fewer where the budget left by the
        pools that cannot be evicted (running, or holding a request) does not
        hold them; None while those pools leave no room for one slot."""
        pinned = sum(p.bytes for p in self.pools if p.in_flight or any(r is not None for r in p.req))
        slots = self.slots_for(key)
        while slots > 1 and pinned + self.footprint(key, slots) > self.budget:
            slots -= 1
        need = self.footprint(key, slots)
        if pinned + need > self.budget:
            return None
        while self.used + need > self.budget:
            # evict an idle, empty pool (the least useful memory first: largest)
            empty = [p for p in self.pools if not p.in_flight and all(r is None for r in p.req)]
            if not empty:
                return None
            victim = max(empty, key=lambda p: p.bytes)
            victim.close()
            self.pools.remove(victim)
            self.stats["pools_evicted"] += 1
        pool = _Pool(self, key, slots)
        if self.tile is not None:
            pool.stepper.select_tile(self.tile)
        self.pools.append(pool)
        self.stats["pools_created"] += 1
        return pool

    def prepare(self, keys):
        """Warm-up before a stream: geometry, dt and one pool per group, each
        stepped once on a stand-in state so that autotuning and graph capture
        happen here and not inside a request's latency."""
        for key in keys:
            if any(p.key == key for p in self.pools):
                continue
            pool = self._new_pool(key)
            if pool is None:
                continue
            _stand_in(pool.stepper, self, key)
            pool.stepper.set_active([0])
            pool.stepper.step(1)
            pool.stepper.set_active([])
            pool.device_active = []

    def close(self):
        for p in self.pools:
            p.close()
        self.pools = []

    def _admit(self, req, now):
        key = req.key
        group = [p for p in self.pools if p.key == key]
        for p in group:
            if not p.in_flight:
                s = p.free_slot()
                if s is not None:
                    return self._place(p, s, req, now)
        if any(p.free_slot() is not None for p in group):
            return False  # a busy pool of the group has room: take it when its chunk ends
        p = self._new_pool(key)
        if p is None:
            return False
        return self._place(p, 0, req, now)

    def _place(self, pool, s, req, now):
        _load(pool.stepper, s, req)
        pool.req[s] = req
        pool.left[s] = self.nsteps(req)
        pool.admitted[s] = now
        pool.active.append(s)
        return True

    def _chunk(self, pool):
        left = min(pool.left[s] for s in pool.active)
        if pool.ms_per_step is None:
            # first chunk of the pool: ~0.13 ns per point and step for one member (B200, MCV4 Nc=256)
            n = 6 * (pool.key[1] * (pool.key[0] - 1) + 1) ** 2
            est = max(1.3e-7 * n * len(pool.active), 0.02)
        else:
            est = pool.ms_per_step
        return max(1, min(left, int(self.chunk_ms / est)))

    def _finish_chunk(self, pool, t, results):
        steps = pool.in_flight
        pool.in_flight = 0
        self.stats["chunks"] += 1
        el = (t - pool.launched) * 1e3 / steps
        pool.ms_per_step = el if pool.ms_per_step is None else 0.5 * (pool.ms_per_step + el)
        for s in pool.active:
            pool.left[s] -= steps
        done = [s for s in pool.active if pool.left[s] == 0]
        if not done:
            return
        flags = pool.stepper.check_finite()
        for s in done:
            req = pool.req[s]
            state = pool.stepper.get_state(s)
            res = Result(req.id, req.order, req.nc, self.nsteps(req), pool.dt, req.arrival, pool.admitted[s],
                         self.clock() - self._t0, finite=not bool(flags[s]),
                         state=state if self.keep_states else None)
            results[req.id] = res
            pool.req[s] = None
        pool.active = [s for s in pool.active if pool.left[s] > 0]

    def run(self, requests):
        """Serve `requests` (arrival times relative to now); returns their Results in input order."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting = []
        results = {}
        self._t0 = self.clock()
        while len(results) < len(requests):
            now = self.clock() - self._t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            progressed = False
            for p in self.pools:
                if p.in_flight and p.stepper.query():
                    self._finish_chunk(p, self.clock() - self._t0, results)
                    progressed = True
            still = []
            for r in waiting:
                if self._admit(r, self.clock() - self._t0):
                    progressed = True
                else:
                    still.append(r)
            waiting = still
            for p in self.pools:
                if not p.in_flight and p.active:
                    if p.device_active != p.active:
                        p.stepper.set_active(p.active)
                        p.device_active = list(p.active)
                    k = self._chunk(p)
                    p.launched = self.clock() - self._t0
                    p.stepper.step_async(k)
                    p.in_flight = k
                    progressed = True
            busy = sum(1 for p in self.pools if p.in_flight)
            self.stats["max_concurrent_pools"] = max(self.stats["max_concurrent_pools"], busy)
            if not progressed:
                if not busy and pending and not waiting:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (self.clock() - self._t0))))
                else:
                    time.sleep(self.poll_s)
        return [results[r.id] for r in requests]


def _load(stepper, slot, req):
    """A request's initial state into a member slot: its host arrays, or its
    spec generated on the device."""
    if req.spec is not None:
        stepper.set_member_balanced_flow(slot, req.spec)
    else:
        stepper.set_member(slot, req.phi_s, req.u, req.v, req.phi)


def _stand_in(stepper, server, key):
    """A plain balanced flow in member 0 (warm-up before a stream)."""
    if server.device_setup:
        stepper.set_member_balanced_flow(0, cases.balanced_flow_spec(cases._Radius(server.radius),
                                                                     np.random.default_rng(0), lmax=0))
        return
    g = server.geometry(key)
    zw, mw, phi, phis, _ = cases.balanced_flow(g, np.random.default_rng(0), lmax=0)
    u, v = api.sphere_to_cov(g, zw, mw)
    stepper.set_member(0, phis, u, v, phi)


def run_one_at_a_time(requests, precision="fp64", scheme="RK3_TVD", radius=cases.EARTH_RADIUS, geoms=None,
                      keep_states=False, tile=None, clock=time.perf_counter, device_setup=False):
    """The plain loop: requests in arrival order, one at a time, each on a
    single-member handle of its grid (handles are created and tuned before the
    stream starts, as the server's are; `tile` pins the stage-kernel shape)."""
    srv = ForecastServer(precision=precision, scheme=scheme, hbm_budget=1 << 62, radius=radius, geoms=geoms,
                         device_setup=device_setup)
    steppers = {}
    for r in requests:
        if r.key not in steppers:
            s = api.Stepper(r.order, r.nc, srv.group_dt(r.key), scheme, members=1, precision=precision, radius=radius)
            if device_setup:
                s.set_geometry_equiangular()
            else:
                s.set_geometry(srv.geometry(r.key))
            if tile is not None:
                s.select_tile(tile)
            _stand_in(s, srv, r.key)
            s.step(1)
            steppers[r.key] = s
    out = {}
    t0 = clock()
    for r in sorted(requests, key=lambda q: q.arrival):
        now = clock() - t0
        if now < r.arrival:
            time.sleep(r.arrival - now)
        s = steppers[r.key]
        admitted = clock() - t0
        n = srv.nsteps(r)
        _load(s, 0, r)
        s.step(n)
        flags = s.check_finite()
        state = s.get_state(0)
        out[r.id] = Result(r.id, r.order, r.nc, n, srv.group_dt(r.key), r.arrival, admitted, clock() - t0,
                           finite=not bool(flags[0]), state=state if keep_states else None)
    for s in steppers.values():
        s.close()
    return [out[r.id] for r in requests]


def run_native(requests, precision="mixed", scheme="RK3_TVD", radius=cases.EARTH_RADIUS, tile=-1, chunk_ms=25.0,
               hbm_budget=0, slot_bytes=8e9, max_slots=32, keep_states=False, geoms=None, prepare=True,
               poll_s=2e-4, clock=time.perf_counter, grouping=None, stats_out=None):
    """Serve `requests` with the native server (mcv_server_*): each request is
    submitted at its arrival time, with the dt and step count ForecastServer
    gives it, and the loop polls until every forecast is back.  grouping:
    (max_grids, max_cost_ratio) of mcv_server_set_grouping, or None (off).  Returns the
    Results in input order (`admitted` is the submission time) and the
    largest number of pools seen with a chunk on the GPU at once."""
    policy = ForecastServer(precision=precision, scheme=scheme, hbm_budget=1 << 62, radius=radius, geoms=geoms)
    results, by_id, busy_max = {}, {}, 0
    with api.Server(precision, scheme, radius, int(hbm_budget), int(slot_bytes), max_slots, chunk_ms, tile) as srv:
        if grouping:
            srv.set_grouping(*grouping)
        if prepare:
            for key in sorted({r.key for r in requests}):
                srv.prepare(key[0], key[1], policy.group_dt(key))
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = clock()
        while len(results) < len(requests):
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                n, dt = policy.nsteps(r), policy.group_dt(r.key)
                if r.spec is not None:
                    rid = srv.submit_spec(r.order, r.nc, dt, n, r.spec)
                else:
                    rid = srv.submit(r.order, r.nc, dt, n, r.phi_s, r.u, r.v, r.phi)
                by_id[rid] = (r, now, dt)
            done = srv.poll()
            busy_max = max(busy_max, srv.stats()["busy_pools"])
            for rid in done:
                r, submitted, dt = by_id.pop(rid)
                state, steps, finite = srv.result(rid)
                results[r.id] = Result(r.id, r.order, r.nc, steps, dt, r.arrival, submitted, clock() - t0,
                                       finite=finite, state=state if keep_states else None)
            if not done:
                if not by_id and pending:
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - (clock() - t0))))
                else:
                    time.sleep(poll_s)
        if stats_out is not None:
            stats_out.update(srv.stats())
            if grouping:
                stats_out["grouped_chunks"] = srv.set_grouping(*grouping)
    return [results[r.id] for r in requests], busy_max


def summarize(results):
    lat = np.array([r.latency for r in results])
    days = sum(r.sim_days for r in results)
    makespan = max(r.finished for r in results) - min(r.arrival for r in results)
    return {"requests": len(results), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
            "sim_days": float(days), "makespan_s": float(makespan), "sim_days_per_s": float(days / makespan),
            "all_finite": all(r.finite for r in results),
            "nonfinite_ids": [int(r.id) for r in results if not r.finite]}
