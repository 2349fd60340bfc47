"""Host logic of the request loop (admission by footprint, chunking, slot
reuse, eviction) with a stand-in for the device handle: each member's "state"
counts the steps it was advanced, so a forecast that is stepped too far or
too little shows up exactly."""
import os

import numpy as np
import pytest

from mcv_sw_b200 import api, serving


class FakeStepper:
    """Device handle stand-in: a chunk completes after two polls."""
    created = []

    def __init__(self, order, nc, dt, scheme, members=1, precision="mixed", radius=1.0):
        self.members = members
        self.steps = np.zeros(members, dtype=np.int64)
        self.seed = np.full(members, -1.0)
        self.active = list(range(members))
        self.busy = 0
        self.closed = False
        FakeStepper.created.append(self)

    def set_geometry(self, geom):
        pass

    def select_tile(self, i):
        pass

    def set_geometry_equiangular(self):
        self.device_geometry = True

    def set_member_balanced_flow(self, m, spec):
        assert not self.busy, "member upload while a chunk is in flight"
        self.seed[m] = spec["marker"]
        self.steps[m] = 0

    def set_member(self, m, phi_s, u, v, phi):
        assert not self.busy, "member upload while a chunk is in flight"
        self.seed[m] = phi.flat[0]
        self.steps[m] = 0

    def set_active(self, members):
        assert not self.busy, "active set changed while a chunk is in flight"
        assert len(set(members)) == len(members)
        self.active = list(members)

    def step_async(self, k):
        assert not self.busy and k >= 1
        self.busy = 2
        self.pending = k

    def step(self, k):
        self.step_async(k)
        while not self.query():
            pass

    def query(self):
        if self.busy:
            self.busy -= 1
            if self.busy == 0:
                for m in self.active:
                    self.steps[m] += self.pending
        return self.busy == 0

    def check_finite(self):
        assert not self.busy
        return np.zeros(self.members, dtype=bool)

    def get_state(self, m):
        assert not self.busy
        return {"seed": self.seed[m], "steps": int(self.steps[m])}

    def close(self):
        self.closed = True


def fake_footprint(order, nc, scheme, precision, members):
    return (1000 + 100 * members) * nc


def requests(specs):
    out = []
    for i, (t, order, nc, hours) in enumerate(specs):
        phi = np.full((6, 4, 4), float(i))
        out.append(serving.Request(i, t, order, nc, hours, phi * 0, phi * 0, phi * 0, phi))
    return out


def server(**kw):
    FakeStepper.created = []
    kw.setdefault("hbm_budget", 10 ** 9)
    return serving.ForecastServer(stepper_factory=FakeStepper, footprint_fn=fake_footprint, keep_states=True,
                                  poll_s=0.0, slot_bytes=300 * 8, chunk_ms=1e-3, **kw)


def test_every_request_gets_exactly_its_steps():
    reqs = requests([(0.0, 3, 8, 2.0), (0.0, 3, 8, 5.0), (0.001, 4, 8, 3.0), (0.002, 3, 8, 1.0),
                     (0.002, 3, 12, 4.0), (0.003, 4, 8, 6.0), (0.003, 3, 8, 2.5)])
    srv = server()
    res = srv.run(reqs)
    assert [r.id for r in res] == [q.id for q in reqs]
    for q, r in zip(reqs, res):
        assert r.state["seed"] == q.phi.flat[0]  # its own slot
        assert r.state["steps"] == r.nsteps == srv.nsteps(q)
        assert r.finished >= r.admitted >= r.arrival
    # 3 slots per (3, 8) pool (slot_bytes / per-member bytes): one or two pools
    # for its four requests (a slot may free up before the fourth arrives), one
    # each for (4, 8) and (3, 12)
    assert 3 <= srv.stats["pools_created"] <= 4


def test_slots_are_reused_and_pools_added_when_full():
    # slot_bytes 300*8 with footprint 100*nc per member -> 3 slots per pool at nc=8
    reqs = requests([(0.0, 3, 8, 1.0 + k) for k in range(7)])
    srv = server()
    res = srv.run(reqs)
    assert all(r.state["steps"] == r.nsteps for r in res)
    assert srv.stats["pools_created"] == 3  # 7 concurrent requests / 3 slots
    assert srv.slots_for((3, 8)) == 3


def test_admission_waits_for_budget_and_evicts_idle_pools():
    # budget for one pool only: the Nc=12 request waits until the Nc=8 pool has
    # drained, which is then evicted to make room
    one = fake_footprint(3, 12, None, None, 3)
    reqs = requests([(0.0, 3, 8, 3.0), (0.0, 3, 12, 1.0)])
    srv = server(hbm_budget=one)
    res = srv.run(reqs)
    assert all(r.state["steps"] == r.nsteps for r in res)
    assert res[1].admitted >= res[0].finished - 1e-9
    assert srv.stats["pools_evicted"] == 1
    assert FakeStepper.created[0].closed


def test_pool_sized_to_the_budget_when_slot_bytes_allow_more():
    # slot_bytes would give max_slots slots, the budget holds one member: the
    # pool is made with one slot and the requests are served one at a time
    FakeStepper.created = []
    reqs = requests([(0.0, 3, 8, 1.0 + k) for k in range(3)])
    srv = serving.ForecastServer(stepper_factory=FakeStepper, footprint_fn=fake_footprint, keep_states=True,
                                 poll_s=0.0, slot_bytes=10 ** 12, chunk_ms=1e-3,
                                 hbm_budget=fake_footprint(3, 8, None, None, 1))
    res = srv.run(reqs)
    assert all(r.state["steps"] == r.nsteps for r in res)
    assert srv.stats["pools_created"] == 1 and FakeStepper.created[0].members == 1


def test_summary():
    reqs = requests([(0.0, 3, 8, 2.0), (0.0, 3, 8, 4.0)])
    s = serving.summarize(server().run(reqs))
    assert s["requests"] == 2 and s["all_finite"]
    assert s["p99_latency_s"] >= s["p50_latency_s"] > 0
    assert s["sim_days_per_s"] > 0


def test_request_stream_matches_configuration():
    reqs = serving.cases.serving_requests(seed=4, count=400)
    t = np.array([r["t"] for r in reqs])
    assert np.all(np.diff(t) > 0)
    assert abs(len(reqs) / t[-1] - 20.0) < 3.0  # Poisson rate 20/s
    ncs = np.array([r["nc"] for r in reqs])
    for nc, p in ((48, 0.4), (96, 0.3), (192, 0.2), (384, 0.1)):
        assert abs(np.mean(ncs == nc) - p) < 0.07
    hours = np.array([r["hours"] for r in reqs])
    assert hours.min() >= 6.0 and hours.max() <= 120.0
    assert abs(np.mean([r["order"] == 3 for r in reqs]) - 0.5) < 0.08
    assert abs(np.mean([r["mountain"] for r in reqs]) - 0.5) < 0.08


@pytest.mark.parametrize("order,nc", [(3, 8), (4, 12)])
def test_serving_dt_is_below_the_cfl_limit(order, nc):
    from mcv_sw_b200 import api, cases
    g = api.Geometry(order, nc, cases.EARTH_RADIUS)
    dt = cases.serving_dt(g)
    for seed in range(3):
        st = cases.serving_state(g, dict(seed=seed, mountain=bool(seed % 2), hours=6.0))
        assert dt <= cases.cfl_dt(g, st.u, st.v, st.phi, 0.5)


def test_device_setup_admits_spec_requests():
    """device_setup: pools take their geometry on the device and requests that
    carry a spec are loaded by generating their state there."""
    specs = [(0.0, 3, 8, 2.0), (0.0, 3, 8, 3.0), (0.001, 4, 8, 1.0), (0.002, 3, 8, 4.0)]
    reqs = [serving.Request(i, t, o, nc, h, spec={"marker": 100.0 + i}) for i, (t, o, nc, h) in enumerate(specs)]
    srv = server(device_setup=True)
    res = srv.run(reqs)
    for q, r in zip(reqs, res):
        assert r.state["seed"] == q.spec["marker"]
        assert r.state["steps"] == r.nsteps == srv.nsteps(q)
    assert all(getattr(st, "device_geometry", False) for st in FakeStepper.created)


def test_native_server_arguments_and_queue():
    """mcv_server_*: argument checks and the request queue, before any device
    call (admission, which creates pools, happens only in mcv_server_poll)."""
    L = api.lib()
    with pytest.raises(api.MCVError) as e:
        api.Server("fp64", hbm_budget=1 << 30, chunk_ms=0.0)
    assert e.value.code == -1
    with pytest.raises(api.MCVError) as e:
        api.Server("fp64", hbm_budget=1 << 30, tile=-2)
    assert e.value.code == -1
    with api.Server("fp64", hbm_budget=1 << 30) as srv:
        assert srv.poll() == []
        npx, _, _ = api.grid_sizes(3, 4)
        z = np.zeros((6, npx, npx))
        for order, nc, dt, n in ((3, 1, 100.0, 1), (3, 4, -1.0, 1), (3, 4, float("nan"), 1), (3, 4, 100.0, 0)):
            with pytest.raises(api.MCVError) as e:
                srv.submit(order, nc, dt, n, z, z, z, z)
            assert e.value.code == -1
        with pytest.raises(ValueError):
            srv.submit(3, 4, 100.0, 1, z[:3], z, z, z)
        assert srv.submit(3, 4, 100.0, 2, z, z, z, z) == 1
        assert srv.submit_spec(4, 4, 50.0, 3, {"gh0": 2.94e4, "u0": 10.0, "alpha": 0.0, "lmax": 0, "rms": 0.0,
                                                "coef": None, "mountain": None}) == 2
        st = srv.stats()
        assert (st["waiting"], st["running"], st["pools"], st["pool_bytes"]) == (2, 0, 0, 0)
        assert srv.result(1) is None  # queued
        assert L.mcv_server_result(srv.s, 99, None, None, None, None, None, None) == -1
        assert L.mcv_server_submit_balanced_flow(srv.s, 3, 4, 100.0, 1, 2.94e4, 0.0, 0.0, 2, None, 1.0, 0.0, 0.0,
                                                 0.0, 0.0, None) == -1
    with api.Server("fp64", hbm_budget=1000) as tiny:
        with pytest.raises(api.MCVError) as e:
            tiny.submit(3, 4, 100.0, 1, z, z, z, z)
        assert e.value.code == -3  # even a one-slot pool exceeds the budget


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU behaviour")
def test_native_server_has_no_cpu_path():
    npx, _, _ = api.grid_sizes(3, 4)
    z = np.zeros((6, npx, npx))
    with api.Server("fp64", hbm_budget=1 << 30) as srv:
        srv.submit(3, 4, 100.0, 2, z, z, z, z)
        with pytest.raises(api.MCVError) as e:
            srv.poll()  # admission creates the pool's handle
        assert e.value.code == -2
