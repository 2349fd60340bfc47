"""Shared helpers of the parity tests."""
import numpy as np

GRAVITY = 9.80616
FILL = -9999999999999999.0


def rel_l2(a, b):
    d = np.sqrt(np.sum((np.asarray(a) - np.asarray(b)) ** 2))
    r = np.sqrt(np.sum(np.asarray(b) ** 2))
    return float(d / r) if r > 0 else float(d)


def interior(a, H, n):
    return a[..., H:H + n, H:H + n]


def halo_strips(a, H, n):
    """The four non-corner halo strips of a padded field (6, npx, npx)."""
    return np.concatenate([
        a[:, H:H + n, 0:H].ravel(), a[:, H:H + n, H + n:].ravel(),
        a[:, 0:H, H:H + n].ravel(), a[:, H + n:, H:H + n].ravel()])


def oracle_for(state, radius=6.371e6):
    from oracle.oracle import Oracle
    o = Oracle(state.order, state.nc, state.dt, state.scheme, radius)
    o.set_phi_s(state.phi_s)
    o.init_state(state.zonal, state.merid, state.phi)
    return o
