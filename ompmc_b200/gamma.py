"""Gamma index (Low et al., Med. Phys. 25 (1998) 656) on rectilinear voxel
grids, the dose-comparison criterion ompMC's users apply to dose
distributions (2 %/2 mm global).

For each reference voxel centre r_i whose dose is at least `cutoff` x the
normalisation dose, gamma_i = min over positions r within `dta` of r_i of

    sqrt(|r - r_i|^2 / dta^2 + (D_eval(r) - D_ref(r_i))^2 / (dd * D_norm)^2)

with D_eval trilinearly interpolated between evaluated voxel centres and
D_norm the reference maximum (global criterion).  Positions are searched on
a cubic lattice of `dta / steps` spacing inside the sphere of radius `dta`
(only values <= 1 decide pass/fail, so nothing beyond `dta` is needed).
A point passes when gamma_i <= 1.
"""
from __future__ import annotations

import numpy as np

__all__ = ["gamma_index", "gamma_pass_rate"]


def _centres(b):
    b = np.asarray(b, dtype=np.float64)
    return 0.5 * (b[:-1] + b[1:])


def _locate(c, x):
    """Index i and weight t of x between centres c[i], c[i+1] (clamped)."""
    if len(c) == 1:
        return np.zeros(x.shape, dtype=np.int64), np.zeros(x.shape)
    i = np.clip(np.searchsorted(c, x) - 1, 0, len(c) - 2)
    t = np.clip((x - c[i]) / (c[i + 1] - c[i]), 0.0, 1.0)
    return i, t


def _trilinear(d, cx, cy, cz, x, y, z):
    """d indexed [k, j, i] (z, y, x) at voxel centres cx, cy, cz."""
    i, tx = _locate(cx, x)
    j, ty = _locate(cy, y)
    k, tz = _locate(cz, z)
    nx, ny, nz = len(cx), len(cy), len(cz)
    i1 = np.minimum(i + 1, nx - 1)
    j1 = np.minimum(j + 1, ny - 1)
    k1 = np.minimum(k + 1, nz - 1)
    c00 = d[k, j, i] * (1 - tx) + d[k, j, i1] * tx
    c01 = d[k, j1, i] * (1 - tx) + d[k, j1, i1] * tx
    c10 = d[k1, j, i] * (1 - tx) + d[k1, j, i1] * tx
    c11 = d[k1, j1, i] * (1 - tx) + d[k1, j1, i1] * tx
    c0 = c00 * (1 - ty) + c01 * ty
    c1 = c10 * (1 - ty) + c11 * ty
    return c0 * (1 - tz) + c1 * tz


def _offsets(dta, steps):
    h = dta / steps
    r = np.arange(-steps, steps + 1) * h
    ox, oy, oz = np.meshgrid(r, r, r, indexing="ij")
    o = np.stack([ox.ravel(), oy.ravel(), oz.ravel()], axis=1)
    d2 = (o ** 2).sum(axis=1)
    o = o[d2 <= dta * dta * (1 + 1e-12)]
    return o[np.argsort((o ** 2).sum(axis=1), kind="stable")]


def gamma_index(ref_idx, ref_dose, eval_dose, bounds, dd=0.02, dta=0.2, d_norm=None, steps=4, chunk=4096):
    """Gamma of reference points against an evaluated distribution.

    ref_idx: flat voxel indices (x fastest) of the reference points;
    ref_dose: their reference doses; eval_dose: the evaluated dose, shape
    (nz, ny, nx); bounds: (xb, yb, zb) voxel boundaries in cm (dta in cm);
    d_norm: normalisation dose (default: max of ref_dose).  Returns gamma per
    reference point (the smallest value found within the search sphere)."""
    xb, yb, zb = bounds
    cx, cy, cz = _centres(xb), _centres(yb), _centres(zb)
    nx, ny, nz = len(cx), len(cy), len(cz)
    eval_dose = np.asarray(eval_dose, dtype=np.float64).reshape(nz, ny, nx)
    ref_idx = np.asarray(ref_idx, dtype=np.int64)
    ref_dose = np.asarray(ref_dose, dtype=np.float64)
    d_norm = float(ref_dose.max()) if d_norm is None else float(d_norm)
    ddn = dd * d_norm
    i = ref_idx % nx
    j = (ref_idx // nx) % ny
    k = ref_idx // (nx * ny)
    px, py, pz = cx[i], cy[j], cz[k]
    offs = _offsets(dta, steps)
    dist2 = (offs ** 2).sum(axis=1) / (dta * dta)
    out = np.empty(len(ref_idx))
    for s in range(0, len(ref_idx), chunk):
        sl = slice(s, s + chunk)
        qx, qy, qz, qd = px[sl], py[sl], pz[sl], ref_dose[sl]
        best = np.full(len(qx), np.inf)
        for o, w in zip(offs, dist2):
            # offsets come nearest first: a point whose best value is <= w
            # cannot improve any more
            act = np.flatnonzero(best > w)
            if len(act) == 0:
                break
            de = _trilinear(eval_dose, cx, cy, cz, qx[act] + o[0], qy[act] + o[1], qz[act] + o[2]) - qd[act]
            best[act] = np.minimum(best[act], w + (de / ddn) ** 2)
        out[sl] = np.sqrt(best)
    return out


def gamma_pass_rate(ref_idx, ref_dose, eval_dose, bounds, dd=0.02, dta=0.2, cutoff=0.1, d_norm=None, steps=4):
    """Fraction of reference points above `cutoff` x D_norm with gamma <= 1,
    and the gamma values of those points."""
    ref_dose = np.asarray(ref_dose, dtype=np.float64)
    d_norm = float(ref_dose.max()) if d_norm is None else float(d_norm)
    sel = ref_dose >= cutoff * d_norm
    g = gamma_index(np.asarray(ref_idx)[sel], ref_dose[sel], eval_dose, bounds, dd, dta, d_norm, steps)
    return float(np.mean(g <= 1.0)), g
