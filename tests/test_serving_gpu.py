"""Serving on the GPU: every request's result is the same alone and in the mix.

Tolerance: bit-identical.  A member's arithmetic reads only that member's
data, whatever slot, pool, chunking or concurrent launches it shares.  The
runs pin one stage-kernel tile shape (tile=0): split precision's per-tile
references and the compiler's FMA contraction both depend on the shape.
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases, serving

pytestmark = pytest.mark.gpu

SPECS = [  # (arrival s, order, nc, hours, mountain)
    (0.000, 3, 8, 3.0, False), (0.002, 4, 8, 2.0, True), (0.004, 3, 12, 4.0, True),
    (0.006, 3, 8, 1.0, True), (0.008, 4, 8, 5.0, False), (0.010, 3, 8, 2.0, False),
]


def stream():
    geoms, out = {}, []
    for i, (t, order, nc, hours, mountain) in enumerate(SPECS):
        key = (order, nc)
        geoms.setdefault(key, api.Geometry(order, nc, cases.EARTH_RADIUS))
        st = cases.serving_state(geoms[key], dict(seed=100 + i, mountain=mountain, hours=hours))
        out.append(serving.Request(i, t, order, nc, hours, st.phi_s, st.u, st.v, st.phi))
    return out, geoms


def same(a, b):
    return all(np.array_equal(a.state[k], b.state[k]) for k in ("u", "v", "phi"))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_each_result_is_the_same_alone_and_in_the_mix(precision):
    tile = 0
    reqs, geoms = stream()
    srv = serving.ForecastServer(precision=precision, tile=tile, keep_states=True, geoms=geoms,
                                 hbm_budget=4 << 30, slot_bytes=64 << 20, chunk_ms=0.5)
    mix = srv.run(reqs)
    stats = dict(srv.stats)
    srv.close()
    assert all(r.finite for r in mix)
    assert stats["max_concurrent_pools"] >= 2  # groups overlapped on the GPU
    for req, r in zip(reqs, mix):
        alone = serving.ForecastServer(precision=precision, tile=tile, keep_states=True, geoms=geoms,
                                       hbm_budget=4 << 30, slot_bytes=64 << 20)
        (a,) = alone.run([serving.Request(req.id, 0.0, req.order, req.nc, req.hours, req.phi_s, req.u, req.v,
                                          req.phi)])
        alone.close()
        assert a.nsteps == r.nsteps
        assert same(a, r), req.id


def test_fp64_server_matches_one_at_a_time_and_a_plain_handle():
    reqs, geoms = stream()
    srv = serving.ForecastServer(precision="fp64", keep_states=True, geoms=geoms, hbm_budget=4 << 30,
                                 slot_bytes=64 << 20, chunk_ms=0.5, tile=0)
    mix = srv.run(reqs)
    srv.close()
    seq = serving.run_one_at_a_time(reqs, precision="fp64", geoms=geoms, keep_states=True, tile=0)
    for req, a, b in zip(reqs, mix, seq):
        assert same(a, b), req.id
        with api.Stepper(req.order, req.nc, a.dt, "RK3_TVD") as s:
            s.set_geometry(geoms[req.key])
            s.select_tile(0)
            s.set_member(0, req.phi_s, req.u, req.v, req.phi)
            s.step(a.nsteps)
            out = s.get_state(0)
        assert all(np.array_equal(out[k], a.state[k]) for k in ("u", "v", "phi")), req.id


def test_inactive_members_keep_their_state():
    """mcv_set_active: members left out of steps are untouched, also across the
    split-precision buffer swap, and rejoin where they stopped."""
    geom = api.Geometry(4, 8, cases.EARTH_RADIUS)
    st = cases.serving_state(geom, dict(seed=7, mountain=True, hours=1.0))
    dt = cases.serving_dt(geom)
    for precision in ("mixed", "fp64"):
        with api.Stepper(4, 8, dt, "RK3_TVD", members=3, precision=precision, radius=cases.EARTH_RADIUS) as s, \
                api.Stepper(4, 8, dt, "RK3_TVD", members=1, precision=precision, radius=cases.EARTH_RADIUS) as ref:
            s.set_geometry(geom)
            ref.set_geometry(geom)
            s.select_tile(0)
            ref.select_tile(0)
            for m in range(3):
                s.set_member(m, st.phi_s, st.u, st.v, st.phi)
            ref.set_member(0, st.phi_s, st.u, st.v, st.phi)
            s.step(2)
            ref.step(2)
            s.set_active([0, 2])
            s.step(3)
            frozen = s.get_state(1)
            ref2 = ref.get_state(0)
            assert all(np.array_equal(frozen[k], ref2[k]) for k in ("u", "v", "phi"))
            s.set_active([1])
            s.step(3)
            ref.step(3)
            a, b, c = s.get_state(0), s.get_state(1), ref.get_state(0)
            assert all(np.array_equal(a[k], c[k]) for k in ("u", "v", "phi"))
            assert all(np.array_equal(b[k], c[k]) for k in ("u", "v", "phi"))
            s.set_active([])
            s.step(1)  # nothing to advance
            assert not s.check_finite().any()
            assert s.query()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_native_server_matches_the_request_loop(precision):
    """mcv_server_* against ForecastServer with device geometry, on host-array
    and device-generated requests: the same forecasts bit for bit, with pools
    of different grids on the GPU at once."""
    reqs, geoms = stream()
    rng = np.random.default_rng(5)
    for i, (order, nc, hours) in enumerate([(4, 8, 2.0), (3, 12, 1.0)]):
        spec = cases.balanced_flow_spec(cases._Radius(cases.EARTH_RADIUS), rng, lmax=4, mountain=bool(i))
        reqs.append(serving.Request(len(reqs), 0.003 * i, order, nc, hours, spec=spec))
    kw = dict(precision=precision, tile=0, keep_states=True, geoms=geoms, hbm_budget=4 << 30, slot_bytes=64 << 20,
              chunk_ms=0.5)
    py = serving.ForecastServer(device_setup=True, **kw)
    a = py.run(reqs)
    py.close()
    b, busy = serving.run_native(reqs, **kw)
    assert busy >= 2
    for req, x, y in zip(reqs, a, b):
        assert y.finite and x.nsteps == y.nsteps
        assert same(x, y), req.id


def test_device_admission_stream():
    """Requests carrying seeded specs, admitted by generating their states on
    the device into pools whose geometry was built there: each result is the
    same alone and in the mix (split precision), and an FP64 forecast from a
    device-built state matches the same forecast from host arrays to the
    parity bar."""
    reqs, geoms = serving.make_requests(5, seed=11, rate=200.0, specs=True)
    for r in reqs:  # short forecasts on small grids keep the test quick
        r.nc, r.hours = (8 if r.order == 4 else 12), 1.0 + (r.id % 3)
    srv = serving.ForecastServer(precision="mixed", tile=0, keep_states=True, hbm_budget=4 << 30,
                                 slot_bytes=64 << 20, chunk_ms=0.5, device_setup=True)
    mix = srv.run(reqs)
    srv.close()
    assert all(r.finite for r in mix)
    for req, r in zip(reqs, mix):
        alone = serving.ForecastServer(precision="mixed", tile=0, keep_states=True, hbm_budget=4 << 30,
                                       slot_bytes=64 << 20, device_setup=True)
        (a,) = alone.run([serving.Request(req.id, 0.0, req.order, req.nc, req.hours, spec=req.spec)])
        alone.close()
        assert same(a, r), req.id
    req = reqs[0]
    dev = serving.run_one_at_a_time([req], precision="fp64", keep_states=True, device_setup=True)[0]
    geom = api.Geometry(req.order, req.nc, cases.EARTH_RADIUS)
    zw, mw, phi, phis = cases.balanced_flow_from_spec(geom, req.spec)
    u, v = api.sphere_to_cov(geom, zw, mw)
    host_req = serving.Request(req.id, 0.0, req.order, req.nc, req.hours, phis, u, v, phi)
    host = serving.run_one_at_a_time([host_req], precision="fp64", keep_states=True)[0]
    H, n = geom.H, geom.n
    for k in ("u", "v", "phi"):
        a, b = dev.state[k][:, H:H + n, H:H + n], host.state[k][:, H:H + n, H:H + n]
        assert np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)) <= 1e-12, k


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_grouped_native_server_matches_the_request_loop(precision):
    """With grouping, pools of different Nc advance in one batched launch per
    stage (mcv_group_*); every forecast is still the one the request loop gives
    it on the same tile shape and device-built geometry, bit for bit, and the
    one the native loop gives it without grouping.  Candidate 6 is a persistent
    TMA form for both orders; the requests all arrive at once, so the pools of
    the MCV3 grids (Nc 8 and 12, one size class) start together."""
    reqs, geoms = stream()
    for r in reqs:
        r.arrival = 0.0
    kw = dict(precision=precision, tile=6, keep_states=True, geoms=geoms, hbm_budget=4 << 30,
              slot_bytes=64 << 20, chunk_ms=0.5)
    py = serving.ForecastServer(device_setup=True, **kw)
    a = py.run(reqs)
    py.close()
    plain, _ = serving.run_native(reqs, **kw)
    stats = {}
    b, busy = serving.run_native(reqs, grouping=(4, 16.0), stats_out=stats, **kw)
    assert stats["grouped_chunks"] > 0
    for req, x, y, z in zip(reqs, a, b, plain):
        assert y.finite and x.nsteps == y.nsteps
        assert same(x, y), req.id
        assert same(z, y), req.id
