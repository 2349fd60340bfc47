"""The benchmark's seeded workloads built with the oracle alone.

TEST INFRASTRUCTURE ONLY: used by the CPU reference arm of ``bench.py`` (and
checked against the GPU library's host init chain by the CPU tests).  The mesh
is the oracle's (initMesh restated, src/mesh_mod.F90:57-214), the initial state
comes from the oracle's IC routines (oracle/orc_cases.c) and is projected to
covariant winds by the oracle's own initTestCase step
(src/test_case_mod.F90:30-39), so building a workload maps no GPU library.
The seeded draws (harmonic coefficients, mountain centre, wave amplitudes) are
the ones the product's workloads use, taken in the same order from the same
generators, so both arms time the same inputs.
"""
import ctypes
import math

import numpy as np

from . import oracle as orc

GRAVITY = 9.80616
EARTH_RADIUS = 6.371e6
GH0 = 2.94e4
OMEGA = 7.292e-5

_D = ctypes.POINTER(ctypes.c_double)


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


def equator_gh0(u0, radius=EARTH_RADIUS, mean=GH0):
    """gh0 whose balanced flow has area-mean geopotential `mean` (any tilt)."""
    return mean + (radius * OMEGA * u0 + 0.5 * u0 * u0) / 3.0


def draw_balanced_spec(rng, u0=38.6, alpha=0.05, lmax=8, rms=10.0, mountain=False, radius=EARTH_RADIUS):
    """The seeded parameters of a balanced flow, drawn in a fixed order:
    harmonic coefficients (degrees >= 1), then the mountain summit, uniform in
    longitude and in sin(latitude) within +-20 degrees."""
    spec = {"gh0": equator_gh0(u0, radius), "u0": u0, "alpha": alpha, "lmax": int(lmax), "rms": rms,
            "coef": None, "mountain": None}
    if lmax:
        coef = rng.standard_normal((lmax + 1) ** 2)
        coef[:1] = 0.0
        spec["coef"] = coef
    if mountain:
        lon_c = rng.uniform(0.0, 2.0 * np.pi)
        lat_c = float(np.arcsin(rng.uniform(-np.sin(np.radians(20.0)), np.sin(np.radians(20.0)))))
        spec["mountain"] = {"h0": 2000.0, "efold": 1.0e6, "lon": lon_c, "lat": lat_c}
    return spec


class Workload:
    """An oracle instance holding a workload's initial state, with its dt."""

    def __init__(self, name, order, nc, scheme, radius=EARTH_RADIUS):
        self.name, self.order, self.nc, self.scheme, self.radius = name, order, nc, scheme, radius
        self.o = orc.Oracle(order, nc, 1.0, scheme, radius)
        self.lib = self.o.lib
        self.lon = self.o.mesh("lonP")
        self.lat = self.o.mesh("latP")
        self.sqrtG = self.o.mesh("sqrtG")
        self.npts = self.lon.size
        self.shape = self.lon.shape
        self.H, self.n = self.o.H, self.o.n
        self.dx = (90.0 / nc) * (2.0 * np.arcsin(1.0) / 180.0)

    def pv_weights(self):
        """weightsOnPV summed over the cells sharing each point, normalised per
        direction (mesh_mod.F90:183-203), zero in the halo."""
        D, H = self.order, self.H
        w1 = np.array([1.0, 4.0, 1.0]) / 6.0 if D == 3 else np.array([1.0, 3.0, 3.0, 1.0]) / 8.0
        line = np.zeros(self.shape[1])
        for c in range(self.nc):
            line[H + c * (D - 1): H + c * (D - 1) + D] += w1
        return np.outer(line, line)[None, :, :]

    def area_rms(self, h):
        w = self.pv_weights() * self.sqrtG
        return float(np.sqrt(np.sum(w * h * h) / np.sum(w)))

    def tilted_zonal(self, gh0, u0, alpha):
        zw, mw, phi = (np.empty(self.shape) for _ in range(3))
        self.lib.orc_ic_tilted_zonal(self.npts, _dp(self.lon), _dp(self.lat), self.radius, float(gh0), float(u0),
                                     float(alpha), _dp(zw), _dp(mw), _dp(phi))
        return zw, mw, phi

    def balanced_flow(self, spec):
        zw, mw, phi = self.tilted_zonal(spec["gh0"], spec["u0"], spec["alpha"])
        phis = np.zeros(self.shape)
        if spec["lmax"]:
            h = np.zeros(self.shape)
            coef = np.ascontiguousarray(spec["coef"], dtype=np.float64)
            if self.lib.orc_ic_add_harmonics(self.npts, _dp(self.lon), _dp(self.lat), spec["lmax"], _dp(coef), 1.0,
                                             _dp(h)) != 0:
                raise RuntimeError("harmonics failed")
            phi += GRAVITY * (h * (spec["rms"] / self.area_rms(h)))
        mt = spec["mountain"]
        if mt:
            self.lib.orc_ic_add_mountain(self.npts, _dp(self.lon), _dp(self.lat), self.radius, mt["lon"], mt["lat"],
                                         mt["h0"], mt["efold"], _dp(phi), _dp(phis))
        return zw, mw, phi, phis

    def start(self, zw, mw, phi, phis, seconds=None, nsteps=None, cfl=0.5):
        """Load the state into the oracle and set dt: CFL `cfl` on the PV
        spacing with the two directions' signal speeds summed, shortened so a
        whole number of steps makes `seconds` (or `nsteps` steps of the CFL dt)."""
        self.o.set_phi_s(phis)
        self.o.init_state(zw, mw, phi)
        u, v = self.o.state("u"), self.o.state("v")
        IG = self.o.mesh("matrixIG")
        cu = IG[..., 0, 0] * u + IG[..., 1, 0] * v
        cv = IG[..., 0, 1] * u + IG[..., 1, 1] * v
        sx = np.abs(cu) + np.sqrt(IG[..., 0, 0] * phi)
        sy = np.abs(cv) + np.sqrt(IG[..., 1, 1] * phi)
        H, n = self.H, self.n
        smax = float((sx + sy)[:, H:H + n, H:H + n].max())
        dt = cfl * (self.dx / (self.order - 1)) / smax
        if seconds is not None:
            self.nsteps = int(math.ceil(seconds / dt))
            dt = seconds / self.nsteps
        else:
            self.nsteps = int(nsteps)
        self.dt = dt
        self.o.set_dt(dt)
        return self


def build(name):
    """(Workload, description) of a bench workload: 'large', 'small' or 'stress'."""
    if name == "large":
        w = Workload(name, 4, 256, "RK3_TVD")
        spec = draw_balanced_spec(np.random.default_rng(2), 38.6, 0.05, 32, 20.0, mountain=True)
        w.start(*w.balanced_flow(spec), seconds=5 * 86400.0)
        desc = "MCV4 Nc=256 RK3_TVD, seeded balanced tilted zonal flow + harmonics (deg<=32, RMS 20 m) + 2000 m mountain"
    elif name == "small":
        w = Workload(name, 3, 32, "RK4")
        spec = draw_balanced_spec(np.random.default_rng(1), 38.6, 0.05, 8, 10.0)
        w.start(*w.balanced_flow(spec), seconds=86400.0)
        desc = "MCV3 Nc=32 RK4, seeded balanced tilted zonal flow + harmonics (deg 1-8, RMS 10 m)"
    elif name == "stress":
        w = Workload(name, 4, 1024, "RK4")
        rng = np.random.default_rng(5)
        zw, mw, phi = w.tilted_zonal(equator_gh0(38.6, w.radius), 38.6, 0.05)
        phis = np.zeros(w.shape)
        t = np.linspace(-np.pi / 2, np.pi / 2, 2001)
        for R in range(4, 13):
            amp = rng.uniform(50.0, 200.0)
            c = np.abs(np.cos(t) ** R * ((R * R + 2 * R + 2) - (R + 1) ** 2 * np.cos(t) ** 2)).max()
            K = amp * GRAVITY * (R + 1) * (R + 2) / (2.0 * OMEGA * w.radius ** 2 * c)
            w.lib.orc_ic_add_rossby_wave(w.npts, _dp(w.lon), _dp(w.lat), w.radius, R, float(K), _dp(zw), _dp(mw),
                                         _dp(phi))
        w.start(zw, mw, phi, phis, nsteps=200)
        desc = "MCV4 Nc=1024 RK4, balanced zonal flow + Rossby-Haurwitz waves R=4..12 (50-200 m)"
    else:
        raise KeyError(name)
    return w, desc
