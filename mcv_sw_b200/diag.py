"""Host-side diagnostics on downloaded states.

cell_average restates calc_VIA (src/diag_mod.F90:69-93): the weightsOnPV
quadrature of a cell's DOF x DOF points (mesh_mod.F90:183-203).  The norms are
the area-weighted L1/L2/Linf of doc/orderCheck.m:63-81 on cell averages.
"""
import numpy as np


def cell_average(geom, field):
    """(6, nc, nc) cell averages of a padded field (6, npx, npx)."""
    D, nc, H = geom.order, geom.nc, geom.H
    w1 = np.array([1.0, 4.0, 1.0]) / 6.0 if D == 3 else np.array([1.0, 3.0, 3.0, 1.0]) / 8.0
    out = np.zeros((6, nc, nc))
    for jd in range(D):
        for id_ in range(D):
            out += (w1[jd] * w1[id_]) * field[:, H + jd: H + jd + (D - 1) * nc: D - 1,
                                              H + id_: H + id_ + (D - 1) * nc: D - 1]
    return out


def cell_areas(geom):
    """Cell areas from the sqrtG quadrature (the same weights as the averages)."""
    return cell_average(geom, geom.sqrtG)


def norms(geom, model, ref):
    """Normalized (L1, L2, Linf) of model - ref on cell averages (orderCheck.m:63-81)."""
    a, b, w = cell_average(geom, model), cell_average(geom, ref), cell_areas(geom)
    l1 = np.sum(np.abs(a - b) * w) / np.sum(np.abs(b) * w)
    l2 = np.sqrt(np.sum((a - b) ** 2 * w) / np.sum(b ** 2 * w))
    linf = np.max(np.abs(a - b) * w) / np.max(np.abs(b) * w)
    return float(l1), float(l2), float(linf)
