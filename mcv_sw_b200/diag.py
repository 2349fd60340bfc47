"""Host-side diagnostics on downloaded states.

cell_average restates calc_VIA (src/diag_mod.F90:69-93) with the reference's
weightsOnPV (src/mesh_mod.F90:183-203): the outer product of {1, 4, 1}/36
(MCV3) or {1, 3, 3, 1}/80 (MCV4; its weights sum to 0.8, so its cell
"averages" are 0.8 times the mean, as the reference's are), summed in the
jDOF, iDOF order.  The norms are the areaCell-weighted L1/L2/Linf of
doc/orderCheck.m:63-81 on those cell values; they are relative, so the 0.8
cancels.  The device computes the same (Stepper.get_history,
Stepper.height_error_norms) without downloading the state.
"""
import numpy as np

from . import api


def pv_weights(order):
    """weightsOnPV(iDOF, jDOF) as a (jDOF, iDOF) array."""
    a = np.array([1.0, 4.0, 1.0]) if order == 3 else np.array([1.0, 3.0, 3.0, 1.0])
    return np.outer(a, a) / (36.0 if order == 3 else 80.0)


def cell_average(geom, field):
    """(6, nc, nc) calc_VIA values of a padded field (6, npx, npx)."""
    D, nc, H = geom.order, geom.nc, geom.H
    w = pv_weights(D)
    out = np.zeros((6, nc, nc))
    for jd in range(D):
        for id_ in range(D):
            out = out + w[jd, id_] * field[:, H + jd: H + jd + (D - 1) * nc: D - 1,
                                           H + id_: H + id_ + (D - 1) * nc: D - 1]
    return out


def cell_areas(geom):
    """mesh%areaCell of the inner cells, (6, nc, nc)."""
    return api.cell_areas(geom.nc, geom.radius)[:, 1:-1, 1:-1]


def norms(geom, model, ref):
    """Normalized (L1, L2, Linf) of model - ref on calc_VIA values (orderCheck.m:63-81)."""
    a, b, w = cell_average(geom, model), cell_average(geom, ref), cell_areas(geom)
    l1 = np.sum(np.abs(a - b) * w) / np.sum(np.abs(b) * w)
    l2 = np.sqrt(np.sum((a - b) ** 2 * w) / np.sum(b ** 2 * w))
    linf = np.max(np.abs(a - b) * w) / np.max(np.abs(b) * w)
    return float(l1), float(l2), float(linf)
