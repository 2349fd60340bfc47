"""Seeded synthetic initial states for the benchmark workloads.

The balanced flow's mean geopotential depth is 2.94e4 m^2/s^2 (its equatorial
value gh0 is set so that the area mean is 2.94e4).

Every state is evaluated at each padded point's own lon/lat, halo included, as
initTestCase does (src/test_case_mod.F90:13-49), then projected to covariant
winds with (G IA) (test_case_mod.F90:32-39).  The base flow is the balanced
solid-body zonal flow with a tilted axis (the case-5 formulas,
test_case_mod.F90:118-120, without the mountain); perturbations are seeded real
spherical harmonics rescaled to a stated area-weighted RMS height, Gaussian
mountains (phi_s = g hs, phi -= g hs as in test_case_mod.F90:117-128) and
Rossby-Haurwitz waves (test_case_mod.F90:133-191 with other wave numbers).

Workload sizes follow the project's five configurations:
  small     MCV3, Nc=32,  RK4,  tilted zonal + harmonics deg 1-8 (RMS 10 m), 1 day
  large     MCV4, Nc=256, RK3,  + harmonics deg <=32 (RMS 20 m) + mountain, 5 days
  ensemble  MCV3, Nc=128, RK4,  64 members, harmonics deg <=16 RMS U(5,30) m,
            alpha U[0, pi/2], u0 U[20, 40] m/s, 2 days
  serving   MCV3/MCV4, Nc in {48, 96, 192, 384}, 6-120 h, half with mountains
  stress    MCV4, Nc=1024, RK4, zonal waves R=4..12 (50-200 m), 200 steps
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import api

GRAVITY = 9.80616
EARTH_RADIUS = 6.371e6
GH0 = 2.94e4


@dataclass
class InitialState:
    order: int
    nc: int
    scheme: str
    dt: float
    nsteps: int
    phi_s: np.ndarray
    u: np.ndarray
    v: np.ndarray
    phi: np.ndarray
    zonal: np.ndarray = None
    merid: np.ndarray = None
    meta: dict = field(default_factory=dict)


def area_rms(geom, h):
    """Area-weighted RMS over the sphere with the PV quadrature weights."""
    w = geom.pv_weights() * geom.sqrtG
    return float(np.sqrt(np.sum(w * h * h) / np.sum(w)))


def cfl_dt(geom, u, v, phi, cfl=0.5):
    """dt = cfl * (dx/(D-1)) / max over interior PVs of the two directions'
    signal speeds summed, (|c^1| + sqrt(G^11 phi)) + (|c^2| + sqrt(G^22 phi)):
    the CFL number of a dimension-split explicit scheme in two dimensions.
    (With the larger of the two speeds instead of their sum, dt is ~1.8x
    longer and RK4 runs of jets crossing the cube's corners blow up in FP64.)"""
    IG = geom.matrixIG
    cu = IG[..., 0, 0] * u + IG[..., 1, 0] * v
    cv = IG[..., 0, 1] * u + IG[..., 1, 1] * v
    sx = np.abs(cu) + np.sqrt(IG[..., 0, 0] * phi)
    sy = np.abs(cv) + np.sqrt(IG[..., 1, 1] * phi)
    smax = float(geom.interior(sx + sy).max())
    return cfl * (geom.dx / (geom.order - 1)) / smax


def fit_steps(dt_cfl, seconds):
    """Largest dt <= dt_cfl that divides the run length exactly."""
    nsteps = int(math.ceil(seconds / dt_cfl))
    return seconds / nsteps, nsteps


def finish(geom, zw, mw, phi, phis, scheme, seconds=None, nsteps=None, cfl=0.5, meta=None):
    u, v = api.sphere_to_cov(geom, zw, mw)
    dt_cfl = cfl_dt(geom, u, v, phi, cfl)
    if seconds is not None:
        dt, ns = fit_steps(dt_cfl, seconds)
    else:
        dt, ns = dt_cfl, int(nsteps)
    return InitialState(geom.order, geom.nc, scheme, dt, ns, phis, u, v, phi, zw, mw, meta or {})


def equator_gh0(u0, radius=EARTH_RADIUS, mean=GH0):
    """gh0 of the balanced flow whose area-mean geopotential is `mean`: the flow's
    phi = gh0 - (R Omega u0 + u0^2/2) sin^2(theta') has area mean
    gh0 - (R Omega u0 + u0^2/2)/3 for any tilt."""
    return mean + (radius * 7.292e-5 * u0 + 0.5 * u0 * u0) / 3.0


def balanced_flow_spec(geom, rng, u0=38.6, alpha=0.05, lmax=8, rms=10.0, mountain=False, lmin=1):
    """The seeded parameters of a balanced flow, drawn from rng in a fixed order
    (harmonic coefficients, then the mountain centre): what the host chain
    (balanced_flow_from_spec) and the device generator
    (Stepper.set_member_balanced_flow) build the same state from."""
    spec = {"gh0": equator_gh0(u0, geom.radius), "u0": u0, "alpha": alpha, "lmax": int(lmax), "rms": rms,
            "coef": None, "mountain": None}
    if lmax:
        coef = rng.standard_normal((lmax + 1) ** 2)
        coef[: lmin * lmin] = 0.0
        spec["coef"] = coef
    if mountain:
        # summit uniform in longitude and in sin(latitude) within +-20 degrees:
        # with the ~3000 m mean depth (gh0 = 2.94e4) the balanced flow lowers the
        # free surface poleward, and a 2000 m summit further poleward would pierce
        # it (phi -> 0, sqrt(G^ii phi) undefined) in the reference scheme as well
        lon_c = rng.uniform(0.0, 2.0 * np.pi)
        lat_c = float(np.arcsin(rng.uniform(-np.sin(np.radians(20.0)), np.sin(np.radians(20.0)))))
        spec["mountain"] = {"h0": 2000.0, "efold": 1.0e6, "lon": lon_c, "lat": lat_c}
    return spec


def balanced_flow_from_spec(geom, spec):
    """Host arrays (zonal, meridional, phi, phi_s) of a balanced-flow spec."""
    zw, mw, phi = api.tilted_zonal(geom, spec["gh0"], spec["u0"], spec["alpha"])
    phis = np.zeros(geom.shape)
    if spec["lmax"]:
        h = np.zeros(geom.shape)
        api.add_harmonics(geom, h, spec["coef"], 1.0)
        phi += GRAVITY * (h * (spec["rms"] / area_rms(geom, h)))
    mt = spec["mountain"]
    if mt:
        api.add_mountain(geom, phi, phis, mt["lon"], mt["lat"], mt["h0"], mt["efold"])
    return zw, mw, phi, phis


def balanced_flow(geom, rng, u0=38.6, alpha=0.05, lmax=8, rms=10.0, mountain=False, lmin=1):
    spec = balanced_flow_spec(geom, rng, u0, alpha, lmax, rms, mountain, lmin)
    zw, mw, phi, phis = balanced_flow_from_spec(geom, spec)
    meta = {"u0": u0, "alpha": alpha, "lmax": lmax, "rms_m": rms}
    if spec["mountain"]:
        meta.update(mountain_lon=spec["mountain"]["lon"], mountain_lat=spec["mountain"]["lat"])
    return zw, mw, phi, phis, meta


def small(seed=1, nc=32, order=3, scheme="RK4", days=1.0, geom=None):
    geom = geom or api.Geometry(order, nc, EARTH_RADIUS)
    rng = np.random.default_rng(seed)
    zw, mw, phi, phis, meta = balanced_flow(geom, rng, 38.6, 0.05, 8, 10.0)
    return finish(geom, zw, mw, phi, phis, scheme, seconds=days * 86400.0, meta=meta), geom


def large(seed=2, nc=256, order=4, scheme="RK3_TVD", days=5.0, geom=None):
    geom = geom or api.Geometry(order, nc, EARTH_RADIUS)
    rng = np.random.default_rng(seed)
    zw, mw, phi, phis, meta = balanced_flow(geom, rng, 38.6, 0.05, 32, 20.0, mountain=True)
    return finish(geom, zw, mw, phi, phis, scheme, seconds=days * 86400.0, meta=meta), geom


def ensemble_member(geom, seed, scheme="RK4", days=2.0):
    rng = np.random.default_rng(seed)
    alpha = rng.uniform(0.0, np.pi / 2)
    u0 = rng.uniform(20.0, 40.0)
    rms = rng.uniform(5.0, 30.0)
    zw, mw, phi, phis, meta = balanced_flow(geom, rng, u0, alpha, 16, rms)
    return finish(geom, zw, mw, phi, phis, scheme, seconds=days * 86400.0, meta=meta)


def stress(seed=5, nc=1024, order=4, scheme="RK4", nsteps=200, geom=None):
    """Balanced zonal flow plus seeded linear Rossby waves of zonal wavenumber
    4..12, each with a cos(R lon) height amplitude uniform in 50-200 m."""
    geom = geom or api.Geometry(order, nc, EARTH_RADIUS)
    rng = np.random.default_rng(seed)
    zw, mw, phi = api.tilted_zonal(geom, equator_gh0(38.6, geom.radius), 38.6, 0.05)
    phis = np.zeros(geom.shape)
    waves = []
    t = np.linspace(-np.pi / 2, np.pi / 2, 2001)
    for R in range(4, 13):
        amp = rng.uniform(50.0, 200.0)
        # K giving a height amplitude `amp`: max over latitude of the balanced term
        c = np.abs(np.cos(t) ** R * ((R * R + 2 * R + 2) - (R + 1) ** 2 * np.cos(t) ** 2)).max()
        K = amp * GRAVITY * (R + 1) * (R + 2) / (2.0 * 7.292e-5 * geom.radius ** 2 * c)
        api.add_rossby_wave(geom, zw, mw, phi, R, K)
        waves.append((R, amp))
    return finish(geom, zw, mw, phi, phis, scheme, nsteps=nsteps, meta={"waves": waves}), geom


def area_mean(geom, a):
    w = geom.pv_weights() * geom.sqrtG
    return float(np.sum(w * a) / np.sum(w))


def serving_requests(seed=4, rate=20.0, count=64):
    """Poisson arrivals: (t_arrive, order, nc, hours, mountain, seed)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for k in range(count):
        t += rng.exponential(1.0 / rate)
        order = 3 if rng.uniform() < 0.5 else 4
        nc = int(rng.choice([48, 96, 192, 384], p=[0.4, 0.3, 0.2, 0.1]))
        hours = float(rng.uniform(6.0, 120.0))
        reqs.append(dict(t=t, order=order, nc=nc, hours=hours, mountain=bool(rng.uniform() < 0.5),
                         seed=int(rng.integers(1 << 31)), id=k))
    return reqs


def serving_dt(geom, cfl=0.45):
    """Fixed dt of a serving grid (order, Nc): CFL `cfl` on the unperturbed
    balanced flow (u0 = 38.6 m/s, alpha = 0.05).  A request's harmonics (RMS
    10 m) raise the largest signal speed by far less than the margin to 0.5,
    and a mountain lowers it."""
    zw, mw, phi = api.tilted_zonal(geom, equator_gh0(38.6, geom.radius), 38.6, 0.05)
    u, v = api.sphere_to_cov(geom, zw, mw)
    return cfl_dt(geom, u, v, phi, cfl)


def serving_spec(radius, req):
    """The seeded balanced-flow spec of a serving request (the draws of
    serving_state), for initial states generated on the device."""
    return balanced_flow_spec(_Radius(radius), np.random.default_rng(req["seed"]), 38.6, 0.05, 8, 10.0,
                              mountain=req["mountain"])


class _Radius:
    """Stands in for a geometry where only the radius is read."""

    def __init__(self, radius):
        self.radius = float(radius)


def serving_state(geom, req, scheme="RK3_TVD"):
    rng = np.random.default_rng(req["seed"])
    zw, mw, phi, phis, meta = balanced_flow(geom, rng, 38.6, 0.05, 8, 10.0, mountain=req["mountain"])
    return finish(geom, zw, mw, phi, phis, scheme, seconds=req["hours"] * 3600.0, meta=meta)
