"""ctypes wrapper of the CPU oracle (oracle/mcv_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by the test suite, by ``__graft_entry__.smoke``
and by the CPU-baseline leg of ``bench.py``.  The GPU product never imports it.

Arrays follow the reference's Fortran layout: a padded field is a numpy array of
shape (6, npx, npx) whose C order equals Fortran's (i, j, panel) column-major
order, i.e. ``a[p, j, i]`` with padded indices i, j = 0..npx-1 (reference index
= padded index + ips).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile the oracle with its Makefile (gcc, FP64, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, _I]
    lib.orc_destroy.argtypes = [ctypes.c_void_p]
    lib.orc_sizes.argtypes = [ctypes.c_void_p, _I]
    lib.orc_dx.restype = ctypes.c_double
    lib.orc_dx.argtypes = [ctypes.c_void_p]
    lib.orc_get_mesh.restype = ctypes.c_int
    lib.orc_get_mesh.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    lib.orc_get_ghost_iref.argtypes = [ctypes.c_void_p, _I]
    lib.orc_set_phi_s.argtypes = [ctypes.c_void_p, _D]
    lib.orc_init_state.argtypes = [ctypes.c_void_p, _D, _D, _D]
    lib.orc_set_state_cov.argtypes = [ctypes.c_void_p, _D, _D, _D]
    lib.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.orc_get_state.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    lib.orc_spatial_operator.argtypes = [ctypes.c_void_p, _D, _D, _D]
    lib.orc_update_stat.argtypes = [ctypes.c_void_p, _D, _D, _D, ctypes.c_double]
    lib.orc_correct_bdy_ghost.argtypes = [ctypes.c_void_p]
    lib.orc_polyfit.restype = ctypes.c_double
    lib.orc_polyfit.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
    lib.orc_calc_tendP.argtypes = [ctypes.c_void_p, _D, _D, _D, ctypes.c_double, ctypes.c_double]
    lib.orc_linear_interp.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_int]
    lib.orc_total_mass.restype = ctypes.c_double
    lib.orc_total_mass.argtypes = [ctypes.c_void_p]
    lib.orc_total_energy.restype = ctypes.c_double
    lib.orc_total_energy.argtypes = [ctypes.c_void_p]
    lib.orc_calc_VIA.argtypes = [ctypes.c_void_p, _D, _D]
    lib.orc_set_dt.argtypes = [ctypes.c_void_p, ctypes.c_double]
    lib.orc_history.argtypes = [ctypes.c_void_p] + [_D] * 8
    _L = ctypes.c_long
    lib.orc_ic_tilted_zonal.argtypes = [_L, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, _D, _D, _D]
    lib.orc_ic_add_harmonics.restype = ctypes.c_int
    lib.orc_ic_add_harmonics.argtypes = [_L, _D, _D, ctypes.c_int, _D, ctypes.c_double, _D]
    lib.orc_ic_add_mountain.argtypes = [_L, _D, _D, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, _D, _D]
    lib.orc_ic_add_rossby_wave.argtypes = [_L, _D, _D, ctypes.c_double, ctypes.c_int, ctypes.c_double, _D, _D, _D]
    lib.orc_num_threads.restype = ctypes.c_int
    lib.orc_set_num_threads.argtypes = [ctypes.c_int]
    _lib = lib
    return lib


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_D)


STATE_FIELDS = ("u", "v", "phi", "phiG", "contraU", "contraV", "zonal_wind", "meridional_wind")
MESH_FIELDS = ("xP", "yP", "lonP", "latP", "sqrtG", "f", "phi_s")
MATRIX_FIELDS = ("matrixG", "matrixIG", "matrixA", "matrixIA")


class Oracle:
    """One reference model instance: parameters, mesh, ghost weights, stat/tend slots."""

    def __init__(self, order, nc, dt, scheme="RK3_TVD", radius=6371220.0):
        lib = _load()
        self.lib = lib
        self.order = int(order)
        self.nc = int(nc)
        self.dt = float(dt)
        self.scheme = scheme
        st = ctypes.c_int(0)
        sch = {"RK3_TVD": 3, "RK4": 4}[scheme]
        self.h = lib.orc_create(self.order, 90.0 / self.nc, self.dt, sch, float(radius), ctypes.byref(st))
        if st.value != 0:
            if self.h:
                lib.orc_destroy(self.h)
            self.h = None
            raise RuntimeError(f"oracle init failed with status {st.value}")
        sz = (ctypes.c_int * 5)()
        lib.orc_sizes(self.h, sz)
        self.n, self.H, self.npx, self.Nx, self.ncx = list(sz)
        self.dx = lib.orc_dx(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def pshape(self):
        return (6, self.npx, self.npx)

    def mesh(self, name):
        if name in MESH_FIELDS:
            out = np.empty(self.pshape)
            self.lib.orc_get_mesh(self.h, MESH_FIELDS.index(name), _dp(out))
            return out
        if name in MATRIX_FIELDS:
            out = np.empty(self.pshape + (2, 2))  # [..., b, a] = M(a, b)
            self.lib.orc_get_mesh(self.h, 7 + MATRIX_FIELDS.index(name), _dp(out))
            return out
        if name == "areaCell":
            out = np.empty((6, self.ncx, self.ncx))
            self.lib.orc_get_mesh(self.h, 11, _dp(out))
            return out
        if name == "ghost_coef":
            out = np.empty((self.H, self.n))
            self.lib.orc_get_mesh(self.h, 12, _dp(out))
            return out
        if name == "ghost_X":
            out = np.empty((self.H, self.n))
            self.lib.orc_get_mesh(self.h, 13, _dp(out))
            return out
        if name == "ghost_iref":
            out = np.empty((self.H, self.n), dtype=np.int32)
            self.lib.orc_get_ghost_iref(self.h, out.ctypes.data_as(_I))
            return out
        raise KeyError(name)

    def set_phi_s(self, phi_s):
        self.lib.orc_set_phi_s(self.h, _dp(np.ascontiguousarray(phi_s, dtype=np.float64)))

    def init_state(self, zonal, merid, phi):
        """initTestCase's projection of sphere winds + phi given on all padded points."""
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (zonal, merid, phi)]
        self.lib.orc_init_state(self.h, *[_dp(x) for x in a])

    def set_state_cov(self, u, v, phi):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (u, v, phi)]
        self.lib.orc_set_state_cov(self.h, *[_dp(x) for x in a])

    def set_dt(self, dt):
        self.dt = float(dt)
        self.lib.orc_set_dt(self.h, self.dt)

    def step(self, nsteps=1):
        self.lib.orc_step(self.h, int(nsteps))

    def state(self, name):
        out = np.empty(self.pshape)
        self.lib.orc_get_state(self.h, STATE_FIELDS.index(name), _dp(out))
        return out

    def spatial_operator(self):
        shp = (6, self.n, self.n)
        tp, tu, tv = np.empty(shp), np.empty(shp), np.empty(shp)
        self.lib.orc_spatial_operator(self.h, _dp(tp), _dp(tu), _dp(tv))
        return tp, tu, tv

    def update_stat(self, tphiG, tu, tv, inc_t):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (tphiG, tu, tv)]
        self.lib.orc_update_stat(self.h, *[_dp(x) for x in a], float(inc_t))

    def correct_bdy_ghost(self):
        self.lib.orc_correct_bdy_ghost(self.h)

    def polyfit(self, pv, right):
        pv = np.ascontiguousarray(pv, dtype=np.float64)
        return self.lib.orc_polyfit(self.h, 1 if right else 0, _dp(pv))

    def calc_tendP(self, f, q, eL, eR):
        out = np.empty(self.order)
        f = np.ascontiguousarray(f, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        self.lib.orc_calc_tendP(self.h, _dp(out), _dp(f), _dp(q), float(eL), float(eR))
        return out

    def linear_interp(self, src, h):
        out = np.empty(self.n)
        src = np.ascontiguousarray(src, dtype=np.float64)
        self.lib.orc_linear_interp(self.h, _dp(out), _dp(src), int(h))
        return out

    def total_mass(self):
        return self.lib.orc_total_mass(self.h)

    def total_energy(self):
        return self.lib.orc_total_energy(self.h)

    def calc_VIA(self, field):
        out = np.empty((6, self.ncx, self.ncx))
        self.lib.orc_calc_VIA(self.h, _dp(out), _dp(np.ascontiguousarray(field, dtype=np.float64)))
        return out


    def history(self):
        """The history-output sequence of the reference's time loop
        (MCV_SW.F90:62-67) on the current state: addFillValue, convert_wind_P2SP,
        calc_VIA of u, v, phi.  Returns a dict of padded fields u, v, phi,
        zonal, merid and cell fields uC, vC, phiC of shape (6, Nc+2, Nc+2)
        (halo cells 0)."""
        out = {k: np.empty(self.pshape) for k in ("u", "v", "phi", "zonal", "merid")}
        out.update({k: np.empty((6, self.ncx, self.ncx)) for k in ("uC", "vC", "phiC")})
        self.lib.orc_history(self.h, *[_dp(out[k]) for k in ("u", "v", "phi", "zonal", "merid", "uC", "vC",
                                                             "phiC")])
        return out


def num_threads():
    return _load().orc_num_threads()


def set_num_threads(n):
    _load().orc_set_num_threads(int(n))
