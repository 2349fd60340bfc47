"""ctypes binding of libmcv_gpu.so (include/mcv_gpu.h).

Arrays use the reference's layout: a padded field is a C-contiguous numpy array
of shape (6, npx, npx) -- identical in memory to Fortran's (i, j, panel) with
i fastest -- and a 2x2 matrix field has shape (6, npx, npx, 2, 2) holding
M(a, b) at [..., b-1, a-1] (Fortran's (2, 2, i, j, panel)).

There is no CPU path: loading the library or creating a stepper raises
``MCVError`` when the library is missing or no sm_100 GPU is present.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)

RK3_TVD, RK4 = 3, 4
FP64, MIXED = 0, 1
BUSY, ERR_NONFINITE = 1, -5
SCHEMES = {"RK3_TVD": RK3_TVD, "RK4": RK4}
PRECISIONS = {"fp64": FP64, "mixed": MIXED}

_lib = None


class MCVError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib_path():
    return _build.LIB_PATH


def lib():
    """Load libmcv_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB_PATH
    if not os.path.exists(path):
        raise MCVError(-2, f"{path} is missing: run `python -m mcv_sw_b200.build` (there is no CPU fallback)")
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "mcv_last_error": (ctypes.c_char_p, []),
        "mcv_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.POINTER(vp)]),
        "mcv_set_geometry": (ctypes.c_int, [vp, _D, _D, _D, _D, _D, _D, _I, _D]),
        "mcv_set_geometry_equiangular": (ctypes.c_int, [vp]),
        "mcv_get_geometry": (ctypes.c_int, [vp, _D, _D, _D, _D, _D, _I, _D]),
        "mcv_set_member_balanced_flow": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_double, ctypes.c_int, _D, ctypes.c_double,
                                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                        ctypes.c_double]),
        "mcv_set_member": (ctypes.c_int, [vp, ctypes.c_int, _D, _D, _D, _D]),
        "mcv_set_state": (ctypes.c_int, [vp, ctypes.c_int, _D, _D, _D]),
        "mcv_step": (ctypes.c_int, [vp, ctypes.c_int]),
        "mcv_step_async": (ctypes.c_int, [vp, ctypes.c_int]),
        "mcv_sync": (ctypes.c_int, [vp]),
        "mcv_query": (ctypes.c_int, [vp]),
        "mcv_set_active": (ctypes.c_int, [vp, ctypes.c_int, _I]),
        "mcv_check_finite": (ctypes.c_int, [vp, _I]),
        "mcv_selftest_wait": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, _I, _D]),
        "mcv_get_state": (ctypes.c_int, [vp, ctypes.c_int, _D, _D, _D, _D]),
        "mcv_mass_energy": (ctypes.c_int, [vp, ctypes.c_int, _D, _D]),
        "mcv_get_history": (ctypes.c_int, [vp, ctypes.c_int, _D, _D, _D, _D, _D, _D, _D, _D]),
        "mcv_group_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]),
        "mcv_group_step_async": (ctypes.c_int, [vp, ctypes.c_int]),
        "mcv_group_step": (ctypes.c_int, [vp, ctypes.c_int]),
        "mcv_group_sync": (ctypes.c_int, [vp]),
        "mcv_group_query": (ctypes.c_int, [vp]),
        "mcv_group_time_steps": (ctypes.c_int, [vp, ctypes.c_int, _D]),
        "mcv_group_destroy": (ctypes.c_int, [vp]),
        "mcv_height_error_norms": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_int, _D]),
        "mcv_cell_areas": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, _D]),
        "mcv_destroy": (ctypes.c_int, [vp]),
        "mcv_time_steps": (ctypes.c_int, [vp, ctypes.c_int, _D]),
        "mcv_profile_step": (ctypes.c_int, [vp, ctypes.c_int, _D, _D]),
        "mcv_tuning": (ctypes.c_int, [vp, _I, _I, _I, ctypes.POINTER(ctypes.c_float)]),
        "mcv_select_tile": (ctypes.c_int, [vp, ctypes.c_int]),
        "mcv_mass_energy_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp,
                                                   vp, _D, _D]),
        "mcv_grid_sizes": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _I, _I, _I]),
        "mcv_device_memory": (ctypes.c_int, [ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
        "mcv_footprint_bytes": (ctypes.c_longlong, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_int]),
        "mcv_build_geometry": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, _D, _D, _D, _D, _D, _D,
                                              _D, _D, _I, _D]),
        "mcv_ic_williamson": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong, _D, _D, ctypes.c_double, _D, _D, _D,
                                             _D]),
        "mcv_ic_tilted_zonal": (ctypes.c_int, [ctypes.c_longlong, _D, _D, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, _D, _D, _D]),
        "mcv_ic_add_harmonics": (ctypes.c_int, [ctypes.c_longlong, _D, _D, ctypes.c_int, _D, ctypes.c_double, _D]),
        "mcv_ic_add_mountain": (ctypes.c_int, [ctypes.c_longlong, _D, _D, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_double, _D, _D]),
        "mcv_ic_add_rossby_haurwitz": (ctypes.c_int, [ctypes.c_longlong, _D, _D, ctypes.c_double, ctypes.c_int,
                                                      ctypes.c_double, _D, _D, _D]),
        "mcv_ic_add_rossby_wave": (ctypes.c_int, [ctypes.c_longlong, _D, _D, ctypes.c_double, ctypes.c_int,
                                                  ctypes.c_double, _D, _D, _D]),
        "mcv_sphere_to_cov": (ctypes.c_int, [ctypes.c_longlong, _D, _D, _D, _D, _D, _D]),
        "mcv_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_longlong,
                                             ctypes.c_longlong, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                             ctypes.POINTER(vp)]),
        "mcv_server_submit": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_longlong,
                                             _D, _D, _D, _D, ctypes.POINTER(ctypes.c_longlong)]),
        "mcv_server_submit_balanced_flow": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                           ctypes.c_longlong, ctypes.c_double, ctypes.c_double,
                                                           ctypes.c_double, ctypes.c_int, _D, ctypes.c_double,
                                                           ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                           ctypes.c_double, ctypes.POINTER(ctypes.c_longlong)]),
        "mcv_server_prepare": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
        "mcv_server_poll": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int, _I]),
        "mcv_server_result": (ctypes.c_int, [vp, ctypes.c_longlong, _D, _D, _D, _D,
                                             ctypes.POINTER(ctypes.c_longlong), _I]),
        "mcv_server_stats": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_longlong)]),
        "mcv_server_destroy": (ctypes.c_int, [vp]),
        "mcv_server_set_grouping": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double,
                                                   ctypes.POINTER(ctypes.c_longlong)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise MCVError(rc, lib().mcv_last_error().decode())
    return rc


def _dp(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_D)


def _ip(a):
    if a.dtype != np.int32 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("expected a C-contiguous int32 array")
    return a.ctypes.data_as(_I)


def grid_sizes(order, nc):
    npx, n, h = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().mcv_grid_sizes(int(order), int(nc), ctypes.byref(npx), ctypes.byref(n), ctypes.byref(h)))
    return npx.value, n.value, h.value


def footprint_bytes(order, nc, scheme="RK3_TVD", precision="fp64", members=1):
    return int(lib().mcv_footprint_bytes(int(order), int(nc), SCHEMES[scheme], PRECISIONS[precision], int(members)))


def device_memory():
    """(free, total) bytes of the current device."""
    f, t = ctypes.c_longlong(), ctypes.c_longlong()
    _check(lib().mcv_device_memory(ctypes.byref(f), ctypes.byref(t)))
    return f.value, t.value


class Geometry:
    """initMesh + initGhost on the host (mcv_build_geometry)."""

    def __init__(self, order, nc, radius=6371220.0):
        self.order, self.nc, self.radius = int(order), int(nc), float(radius)
        self.npx, self.n, self.H = grid_sizes(order, nc)
        shp = (6, self.npx, self.npx)
        self.lonP, self.latP, self.sqrtG, self.f = (np.empty(shp) for _ in range(4))
        self.matrixG, self.matrixIG, self.matrixA, self.matrixIA = (np.empty(shp + (2, 2)) for _ in range(4))
        self.ghost_iref = np.empty((self.H, self.n), dtype=np.int32)
        self.ghost_coef = np.empty((self.H, self.n))
        _check(lib().mcv_build_geometry(self.order, self.nc, self.radius, _dp(self.lonP), _dp(self.latP),
                                        _dp(self.sqrtG), _dp(self.matrixG), _dp(self.matrixIG), _dp(self.matrixA),
                                        _dp(self.matrixIA), _dp(self.f), _ip(self.ghost_iref), _dp(self.ghost_coef)))
        self.dx = (90.0 / self.nc) * (2.0 * np.arcsin(1.0) / 180.0)

    @property
    def shape(self):
        return (6, self.npx, self.npx)

    @property
    def npts(self):
        return 6 * self.npx * self.npx

    def interior(self, a):
        H, n = self.H, self.n
        return a[:, H:H + n, H:H + n]

    def pv_weights(self):
        """Quadrature weight of every padded point: weightsOnPV summed over the
        cells that share the point (mesh_mod.F90:183-203), zero in the halo."""
        D = self.order
        w1 = np.array([1.0, 4.0, 1.0]) / 6.0 if D == 3 else np.array([1.0, 3.0, 3.0, 1.0]) / 8.0
        line = np.zeros(self.npx)
        for c in range(self.nc):
            line[self.H + c * (D - 1): self.H + c * (D - 1) + D] += w1
        return np.broadcast_to(np.outer(line, line), self.shape)


def cell_areas(nc, radius):
    """mesh%areaCell: (6, nc+2, nc+2) with zero halo cells."""
    out = np.empty((6, nc + 2, nc + 2))
    _check(lib().mcv_cell_areas(int(nc), float(radius), _dp(out)))
    return out


def selftest_wait(complete, limit_ms):
    """Run the stage kernels' bounded copy wait on an mbarrier that is
    (complete=True) or is never (False) completed: (timed_out, elapsed_ms)."""
    t, ms = ctypes.c_int(), ctypes.c_double()
    _check(lib().mcv_selftest_wait(int(bool(complete)), float(limit_ms), ctypes.byref(t), ctypes.byref(ms)))
    return bool(t.value), ms.value


# ---------------------------------------------------------------- initial conditions
def williamson(geom, case_num):
    shp = geom.shape
    zw, mw, phi, phis = (np.empty(shp) for _ in range(4))
    _check(lib().mcv_ic_williamson(int(case_num), geom.npts, _dp(geom.lonP), _dp(geom.latP), geom.radius, _dp(zw),
                                   _dp(mw), _dp(phi), _dp(phis)))
    return zw, mw, phi, phis


def tilted_zonal(geom, gh0, u0, alpha):
    shp = geom.shape
    zw, mw, phi = (np.empty(shp) for _ in range(3))
    _check(lib().mcv_ic_tilted_zonal(geom.npts, _dp(geom.lonP), _dp(geom.latP), geom.radius, float(gh0), float(u0),
                                     float(alpha), _dp(zw), _dp(mw), _dp(phi)))
    return zw, mw, phi


def add_harmonics(geom, phi, coef, scale=1.0):
    coef = np.ascontiguousarray(coef, dtype=np.float64)
    lmax = int(round(np.sqrt(coef.size))) - 1
    assert (lmax + 1) ** 2 == coef.size
    _check(lib().mcv_ic_add_harmonics(geom.npts, _dp(geom.lonP), _dp(geom.latP), lmax, _dp(coef), float(scale),
                                      _dp(phi)))


def add_mountain(geom, phi, phis, lon_c, lat_c, h0=2000.0, efold=1.0e6):
    _check(lib().mcv_ic_add_mountain(geom.npts, _dp(geom.lonP), _dp(geom.latP), geom.radius, float(lon_c),
                                     float(lat_c), float(h0), float(efold), _dp(phi), _dp(phis)))


def add_rossby_haurwitz(geom, zw, mw, phi, wavenumber, omg):
    _check(lib().mcv_ic_add_rossby_haurwitz(geom.npts, _dp(geom.lonP), _dp(geom.latP), geom.radius, int(wavenumber),
                                            float(omg), _dp(zw), _dp(mw), _dp(phi)))


def add_rossby_wave(geom, zw, mw, phi, wavenumber, K):
    _check(lib().mcv_ic_add_rossby_wave(geom.npts, _dp(geom.lonP), _dp(geom.latP), geom.radius, int(wavenumber),
                                        float(K), _dp(zw), _dp(mw), _dp(phi)))


def sphere_to_cov(geom, zw, mw):
    u, v = np.empty(geom.shape), np.empty(geom.shape)
    _check(lib().mcv_sphere_to_cov(geom.npts, _dp(geom.matrixG), _dp(geom.matrixIA), _dp(zw), _dp(mw), _dp(u),
                                   _dp(v)))
    return u, v


def mass_energy_noalloc(order, nc, members, u, v, phi, phi_s, sqrtG, matrixIG, stream=0):
    """mcv_mass_energy_noalloc on caller-owned device memory: the array arguments
    are device addresses (ints) in the reference's layout.  Returns (mass, energy)
    as lists of `members` floats."""
    mass = (ctypes.c_double * members)()
    energy = (ctypes.c_double * members)()
    _check(lib().mcv_mass_energy_noalloc(int(order), int(nc), int(members), u, v, phi, phi_s, sqrtG, matrixIG,
                                         stream or None, mass, energy))
    return list(mass), list(energy)


# ---------------------------------------------------------------- stepping
class Stepper:
    """One device-resident ensemble of `members` states on one grid."""

    def __init__(self, order, nc, dt, scheme="RK3_TVD", members=1, precision="fp64", radius=6371220.0):
        self.order, self.nc, self.dt, self.scheme = int(order), int(nc), float(dt), scheme
        self.members, self.precision, self.radius = int(members), precision, float(radius)
        self.npx, self.n, self.H = grid_sizes(order, nc)
        h = ctypes.c_void_p()
        _check(lib().mcv_create(self.order, self.nc, SCHEMES[scheme], PRECISIONS[precision], self.dt, float(radius),
                                self.members, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().mcv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_geometry(self, geom):
        _check(lib().mcv_set_geometry(self.h, _dp(geom.sqrtG), _dp(geom.matrixG), _dp(geom.matrixIG),
                                      _dp(geom.matrixA), _dp(geom.matrixIA), _dp(geom.f), _ip(geom.ghost_iref),
                                      _dp(geom.ghost_coef)))

    def set_geometry_equiangular(self):
        """Compute the grid geometry on the device (no host arrays, no upload)."""
        _check(lib().mcv_set_geometry_equiangular(self.h))

    def get_geometry(self):
        """The handle's metric planes (padded, Fortran layout) and ghost weights."""
        shp = (6, self.npx, self.npx)
        out = {k: np.empty(shp) for k in ("sqrtG", "ig11", "ig12", "ig22", "f")}
        nh = (self.order - 1, self.npx - 2 * (self.order - 1))
        out["ghost_iref"] = np.empty(nh, dtype=np.int32)
        out["ghost_coef"] = np.empty(nh)
        _check(lib().mcv_get_geometry(self.h, *[_dp(out[k]) for k in ("sqrtG", "ig11", "ig12", "ig22", "f")],
                                      _ip(out["ghost_iref"]), _dp(out["ghost_coef"])))
        return out

    def set_member_balanced_flow(self, m, spec):
        """Member m's initial state generated on the device from a balanced-flow
        spec (cases.balanced_flow_spec): no host arrays, no upload."""
        lmax = int(spec["lmax"])
        coef = np.ascontiguousarray(spec["coef"], dtype=np.float64) if lmax else None
        mt = spec.get("mountain")
        _check(lib().mcv_set_member_balanced_flow(
            self.h, int(m), float(spec["gh0"]), float(spec["u0"]), float(spec["alpha"]), lmax, _dp(coef),
            float(spec["rms"]), float(mt["h0"]) if mt else 0.0, float(mt["lon"]) if mt else 0.0,
            float(mt["lat"]) if mt else 0.0, float(mt["efold"]) if mt else 1.0))

    def set_member(self, m, phi_s, u, v, phi):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (phi_s, u, v, phi)]
        _check(lib().mcv_set_member(self.h, int(m), *[_dp(x) for x in arrs]))

    def set_state(self, m, u, v, phi):
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (u, v, phi)]
        _check(lib().mcv_set_state(self.h, int(m), *[_dp(x) for x in arrs]))

    def step(self, nsteps=1):
        _check(lib().mcv_step(self.h, int(nsteps)))

    def step_async(self, nsteps=1):
        _check(lib().mcv_step_async(self.h, int(nsteps)))

    def sync(self):
        _check(lib().mcv_sync(self.h))

    def query(self):
        """True when all queued work has finished (never waits)."""
        rc = lib().mcv_query(self.h)
        if rc == BUSY:
            return False
        _check(rc)
        return True

    def set_active(self, members):
        """Members the following steps advance (the others keep their state)."""
        ids = np.ascontiguousarray(np.asarray(list(members), dtype=np.int32))
        _check(lib().mcv_set_active(self.h, len(ids), ids.ctypes.data_as(_I) if len(ids) else None))

    def check_finite(self):
        """Per-member flags, True where the interior u, v or phi holds a NaN or Inf."""
        flags = np.zeros(self.members, dtype=np.int32)
        rc = lib().mcv_check_finite(self.h, flags.ctypes.data_as(_I))
        if rc not in (0, ERR_NONFINITE):
            _check(rc)
        return flags.astype(bool)

    def get_state(self, m=0, out=None):
        shp = (6, self.npx, self.npx)
        out = out or {k: np.empty(shp) for k in ("u", "v", "phi", "phiG")}
        _check(lib().mcv_get_state(self.h, int(m), _dp(out.get("u")), _dp(out.get("v")), _dp(out.get("phi")),
                                   _dp(out.get("phiG"))))
        return out

    def time_steps(self, nsteps):
        """Advance nsteps; device milliseconds (CUDA events on the library stream)."""
        ms = ctypes.c_double()
        _check(lib().mcv_time_steps(self.h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def profile_step(self, nsteps=1):
        """Advance nsteps with per-launch events: (mean ms per stage kernel, mean ms per halo kernel)."""
        st = (ctypes.c_double * 4)()
        ha = ctypes.c_double()
        _check(lib().mcv_profile_step(self.h, int(nsteps), st, ctypes.byref(ha)))
        nst = 3 if self.scheme == "RK3_TVD" else 4
        return list(st)[:nst], ha.value

    def tuning(self):
        """Autotuner record: list of ((cells_x, cells_y, threads, walk, ctas_per_sm, tma), ms per launch)
        and the chosen index."""
        n, ch = ctypes.c_int(), ctypes.c_int()
        shapes = (ctypes.c_int * 96)()
        ms = (ctypes.c_float * 16)()
        _check(lib().mcv_tuning(self.h, ctypes.byref(n), ctypes.byref(ch), shapes, ms))
        cands = [(tuple(shapes[6 * i: 6 * i + 6]), ms[i]) for i in range(n.value)]
        return cands, ch.value

    def select_tile(self, index):
        _check(lib().mcv_select_tile(self.h, int(index)))

    def mass_energy(self, m=0):
        ms, en = ctypes.c_double(), ctypes.c_double()
        _check(lib().mcv_mass_energy(self.h, int(m), ctypes.byref(ms), ctypes.byref(en)))
        return ms.value, en.value

    def get_history(self, m=0, fields=("u", "v", "phi", "zonal", "merid", "uC", "vC", "phiC")):
        """mcv_get_history: the reference's history-output sequence on member m
        (addFillValue, convert_wind_P2SP, calc_VIA of u, v, phi) formed on the
        device.  Padded fields have shape (6, npx, npx), cell fields
        (6, nc+2, nc+2) with zero halo cells."""
        cell = (6, self.nc + 2, self.nc + 2)
        names = ("u", "v", "phi", "zonal", "merid", "uC", "vC", "phiC")
        out = {k: np.empty(cell if k.endswith("C") else (6, self.npx, self.npx)) for k in fields}
        _check(lib().mcv_get_history(self.h, int(m), *[_dp(out.get(k)) for k in names]))
        return out

    def height_error_norms(self, m, ref, ref_m=0):
        """(L1, L2, Linf) of member m's phi against member ref_m of Stepper
        `ref`, on calc_VIA cell averages weighted by areaCell (orderCheck.m)."""
        out = (ctypes.c_double * 3)()
        _check(lib().mcv_height_error_norms(self.h, int(m), ref.h, int(ref_m), out))
        return tuple(out)


class Group:
    """Several Steppers (one order, precision and scheme; any Nc, dt, members)
    advanced together, one batched stage-kernel launch per RK stage
    (mcv_group_*).  tile: the candidate index of the launch, or -1 for the
    first stepper's choice."""

    def __init__(self, steppers, tile=-1):
        self.steppers = list(steppers)
        arr = (ctypes.c_void_p * len(self.steppers))(*[s.h for s in self.steppers])
        g = ctypes.c_void_p()
        _check(lib().mcv_group_create(arr, len(self.steppers), int(tile), ctypes.byref(g)))
        self.g = g

    def step(self, nsteps):
        _check(lib().mcv_group_step(self.g, int(nsteps)))

    def step_async(self, nsteps):
        _check(lib().mcv_group_step_async(self.g, int(nsteps)))

    def sync(self):
        _check(lib().mcv_group_sync(self.g))

    def query(self):
        rc = lib().mcv_group_query(self.g)
        if rc == BUSY:
            return False
        _check(rc)
        return True

    def time_steps(self, nsteps):
        ms = ctypes.c_double()
        _check(lib().mcv_group_time_steps(self.g, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def close(self):
        if getattr(self, "g", None):
            lib().mcv_group_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


SERVER_STATS = ("waiting", "running", "unclaimed", "pools", "busy_pools", "pool_bytes", "pools_created",
                "pools_evicted", "chunks")


class Server:
    """The native forecast server (mcv_server_*): requests are queued with
    submit / submit_spec, mcv_server_poll runs one pass of the request loop,
    and a finished forecast's state is taken with result."""

    def __init__(self, precision="mixed", scheme="RK3_TVD", radius=6371220.0, hbm_budget=0, slot_bytes=8 << 30,
                 max_slots=32, chunk_ms=25.0, tile=-1):
        self.precision, self.scheme, self.radius = precision, scheme, float(radius)
        s = ctypes.c_void_p()
        _check(lib().mcv_server_create(PRECISIONS[precision], SCHEMES[scheme], self.radius, int(hbm_budget),
                                       int(slot_bytes), int(max_slots), float(chunk_ms), int(tile), ctypes.byref(s)))
        self.s = s
        self.grids = {}  # request id -> (order, nc)

    def set_grouping(self, max_grids=4, max_cost_ratio=4.0):
        """Idle pools of one order whose step costs are within max_cost_ratio
        advance together in one batched launch (max_grids pools; 1: off).
        Returns the grouped chunks launched so far."""
        n = ctypes.c_longlong()
        _check(lib().mcv_server_set_grouping(self.s, int(max_grids), float(max_cost_ratio), ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "s", None):
            lib().mcv_server_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, order, nc, dt, nsteps, phi_s, u, v, phi):
        npx, _, _ = grid_sizes(order, nc)
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (phi_s, u, v, phi)]
        if any(a.size != 6 * npx * npx for a in arrs):
            raise ValueError(f"state arrays must hold 6 x {npx} x {npx} points")
        rid = ctypes.c_longlong()
        _check(lib().mcv_server_submit(self.s, int(order), int(nc), float(dt), int(nsteps), *[_dp(x) for x in arrs],
                                       ctypes.byref(rid)))
        self.grids[rid.value] = (int(order), int(nc))
        return rid.value

    def submit_spec(self, order, nc, dt, nsteps, spec):
        """A forecast whose initial state the device generates from a
        balanced-flow spec (cases.balanced_flow_spec) at admission."""
        lmax = int(spec["lmax"])
        coef = np.ascontiguousarray(spec["coef"], dtype=np.float64) if lmax else None
        mt = spec.get("mountain")
        rid = ctypes.c_longlong()
        _check(lib().mcv_server_submit_balanced_flow(
            self.s, int(order), int(nc), float(dt), int(nsteps), float(spec["gh0"]), float(spec["u0"]),
            float(spec["alpha"]), lmax, _dp(coef), float(spec["rms"]), float(mt["h0"]) if mt else 0.0,
            float(mt["lon"]) if mt else 0.0, float(mt["lat"]) if mt else 0.0, float(mt["efold"]) if mt else 1.0,
            ctypes.byref(rid)))
        self.grids[rid.value] = (int(order), int(nc))
        return rid.value

    def prepare(self, order, nc, dt):
        _check(lib().mcv_server_prepare(self.s, int(order), int(nc), float(dt)))

    def poll(self, max_ids=64):
        """One pass of the request loop; ids of the forecasts finished since the last poll."""
        ids = (ctypes.c_longlong * max(1, max_ids))()
        n = ctypes.c_int()
        _check(lib().mcv_server_poll(self.s, ids, int(max_ids), ctypes.byref(n)))
        return list(ids[: n.value])

    def result(self, rid):
        """(state dict u, v, phi, phiG over the padded range, steps taken, finite), or None while running."""
        order, nc = self.grids[rid]
        npx, _, _ = grid_sizes(order, nc)
        out = {k: np.empty((6, npx, npx)) for k in ("u", "v", "phi", "phiG")}
        steps, fin = ctypes.c_longlong(), ctypes.c_int()
        rc = lib().mcv_server_result(self.s, int(rid), *[_dp(out[k]) for k in ("u", "v", "phi", "phiG")],
                                     ctypes.byref(steps), ctypes.byref(fin))
        if rc == BUSY:
            return None
        _check(rc)
        del self.grids[rid]
        return out, steps.value, bool(fin.value)

    def stats(self):
        st = (ctypes.c_longlong * 9)()
        _check(lib().mcv_server_stats(self.s, st))
        return dict(zip(SERVER_STATS, list(st)))
