"""Host mirror of ompMC's matRad MEX entry (ucodes/omc_matrad/omc_matrad.c).

`matrad_dij(cubeRho, cubeMatIx, mcGeo, mcSrc, mcOpt, nargout=1)` takes what
matRad passes to `omc_matrad(...)` (omc_matrad.c:1417 mexFunction), with
Python dicts in place of MATLAB structs and numpy arrays in place of MATLAB
arrays, and returns the dose influence matrix D as a scipy CSC matrix of
shape (number of voxels, number of bixels); with `nargout=2` it also returns
the matrix of variances, like `[D, V] = omc_matrad(...)`.

Input conventions follow the MEX entry:

* `cubeRho` float64 and `cubeMatIx` int32, both 3-D with MATLAB indexing
  (i, j, k) = (x, y, z); voxel n = i + j*nx + k*nx*ny (column-major), which
  is also the row index of D (omc_matrad.c:1590-1640);
* `cubeMatIx` counts media from 1 (omc_matrad.c:1138);
* `mcGeo`: `material` (list of medium names, or a list of rows whose first
  entry is the name, like matRad's cell array), `xBounds`, `yBounds`,
  `zBounds` (nx+1, ny+1, nz+1 voxel boundaries in cm);
* `mcSrc`: `nBixels`, `iBeam` (1-based, per bixel), `xSource`/`ySource`/
  `zSource` (per beam), `xCorner`..`zSide2` (per bixel) (omc_matrad.c:776-832);
* `mcOpt`: `verbose`, `nHistories` (per bixel, default 1e4), `nBatches`
  (default 10), `sourceGeometry` ('point' | 'gaussian'),
  `sourceGaussianWidth` (default 0.2123), `nSplit`, `spectrumFile`
  (default ./spectra/mohan6.spectrum), `monoEnergy` (parsed and unused, as
  in omc_matrad.c:625 which always reads the spectrum), `charge`,
  `global_ecut`, `global_pcut`, `randomSeeds` (two integers), `pegsFile`,
  `pgs4formFile`, `dataFolder`, `outputFolder`, `relDoseThreshold`
  (default 0.01) (omc_matrad.c:137-353).  Two optional fields select how
  the engine runs: `gpuDevice` (default 0) and `transport` ('event', the
  FP32 event-based form, default; 'plain', the FP64 history-based form).

Errors raise `MexError` with the identifier the MEX entry gives
mexErrMsgIdAndTxt.  The random numbers are not RANMAR's: `randomSeeds`
seeds per-bixel Philox streams, so D agrees with the reference within its
statistical uncertainty rather than bit for bit.  Photon splitting
(`nSplit` > 1, ompmc.c:1867-2139) is supported up to nSplit = 64.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .engine import EVENT_FP32, PLAIN_FP64, Engine, Tables, load_spectrum

__all__ = ["MexError", "matrad_dij"]


class MexError(RuntimeError):
    """mexErrMsgIdAndTxt(identifier, message)."""

    def __init__(self, identifier, message):
        super().__init__(f"{identifier}: {message}")
        self.identifier = identifier


class _Cube:
    """Phantom in the engine's layout: arrays indexed [k, j, i]."""

    def __init__(self, media, xb, yb, zb, med, rho):
        self.media, self.xb, self.yb, self.zb, self.med, self.rho = media, xb, yb, zb, med, rho

    @property
    def shape(self):
        return (len(self.xb) - 1, len(self.yb) - 1, len(self.zb) - 1)


_tables: dict = {}


def _tables_for(pegs, pgs4form, data_folder, media):
    key = (str(pegs), str(pgs4form), str(data_folder), tuple(media))
    if key not in _tables:
        _tables[key] = Tables(pegs, pgs4form, data_folder, list(media))
    return _tables[key]


def _field(s, name, default=None, required=False):
    if not isinstance(s, dict):
        return default
    if name in s and s[name] is not None:
        return s[name]
    if required:
        # the MEX entry passes a missing field to num2str / mxArrayToString,
        # which fails (omc_matrad.c:236-340)
        raise MexError("matRad:omc_matrad:Error", f"Call to num2str not successful ({name} missing)")
    return default


def _scalar(v):
    return float(np.asarray(v, dtype=np.float64).ravel()[0])


def _material_names(mat):
    if mat is None:
        raise MexError("matRad:omc_matrad:Error", "No materials specified!")
    names = []
    for m in mat:
        name = m if isinstance(m, str) else (m[0] if len(m) else None)
        if not isinstance(name, str):
            raise MexError("matRad:omc_matrad:Error", "Material string could not be read!")
        names.append(name)
    if not names:
        raise MexError("matRad:omc_matrad:Error", "No materials specified!")
    return names


def _check_inputs(cubeRho, cubeMatIx, mcGeo, mcSrc):
    """Argument checks of parseInput (omc_matrad.c:157-175), in order."""
    if not (isinstance(cubeRho, np.ndarray) and cubeRho.dtype == np.float64):
        raise MexError("matRad:matRad_ompInterface:inputNotDouble", "Input argument must be of type double.")
    if cubeRho.ndim != 3:
        raise MexError("matRad:matRad_ompInterface:inputNot3D", "Input argument 1 must be a three-dimensional cube\n")
    if not (isinstance(cubeMatIx, np.ndarray) and cubeMatIx.dtype == np.int32):
        raise MexError("matRad:matRad_ompInterface:inputNotInt32", "The density cube must be a 32 bit integer array!")
    if not isinstance(mcGeo, dict):
        raise MexError("MATLAB:phonebook:inputNotStruct", "Input 3 must be a mcGeo Structure.")
    if not isinstance(mcSrc, dict):
        raise MexError("MATLAB:phonebook:inputNotStruct", "Input 4 must be a mcSrc Structure.")


def _geometry(cubeRho, cubeMatIx, mcGeo):
    media = _material_names(_field(mcGeo, "material"))
    nx, ny, nz = cubeRho.shape
    if cubeMatIx.shape != cubeRho.shape:
        raise MexError("matRad:omc_matrad:Error", "cubeMatIx and cubeRho differ in shape")
    xb, yb, zb = (np.ascontiguousarray(np.asarray(_field(mcGeo, k, required=True), dtype=np.float64).ravel())
                  for k in ("xBounds", "yBounds", "zBounds"))
    if (len(xb), len(yb), len(zb)) != (nx + 1, ny + 1, nz + 1):
        raise MexError("matRad:omc_matrad:Error", "voxel boundaries do not match the cube size")
    med = np.ascontiguousarray(cubeMatIx.transpose(2, 1, 0))
    if med.min() < 1 or med.max() > len(media):
        raise MexError("matRad:omc_matrad:Error", "material index outside 1..number of materials")
    rho = np.ascontiguousarray(cubeRho.transpose(2, 1, 0))
    return _Cube(media, xb, yb, zb, med, rho)


def _source(mcSrc, mcOpt, cube):
    nbix = int(_scalar(_field(mcSrc, "nBixels", required=True)))
    ibeam = np.asarray(_field(mcSrc, "iBeam", required=True), dtype=np.float64).ravel()[:nbix].astype(np.int32) - 1
    per_beam = [np.asarray(_field(mcSrc, k, required=True), dtype=np.float64).ravel()
                for k in ("xSource", "ySource", "zSource")]
    nbeams = int(ibeam.max()) + 1 if nbix else 0
    if ibeam.size != nbix or ibeam.min(initial=0) < 0 or any(len(a) < nbeams for a in per_beam):
        raise MexError("matRad:omc_matrad:Error", "iBeam / source position arrays are inconsistent")
    per_bix = {}
    for name in ("Corner", "Side1", "Side2"):
        cols = [np.asarray(_field(mcSrc, a + name, required=True), dtype=np.float64).ravel() for a in "xyz"]
        if any(len(c) < nbix for c in cols):
            raise MexError("matRad:omc_matrad:Error", f"{name} arrays shorter than nBixels")
        per_bix[name] = np.stack([c[:nbix] for c in cols], axis=1)
    spectrum_file = str(_field(mcOpt, "spectrumFile", "./spectra/mohan6.spectrum"))
    if not Path(spectrum_file).is_file():
        raise MexError("matRad:omc_matrad:Error", f"Unable to open file: {spectrum_file}")
    geo = str(_field(mcOpt, "sourceGeometry", "point"))
    bl = dict(src=np.stack([a[:nbeams] for a in per_beam], axis=1), corner=per_bix["Corner"],
              side1=per_bix["Side1"], side2=per_bix["Side2"], ibeam=ibeam,
              spectrum=load_spectrum(spectrum_file), charge=int(_scalar(_field(mcOpt, "charge", required=True))),
              gaussian=(geo == "gaussian"),
              gauss_width=float(_scalar(_field(mcOpt, "sourceGaussianWidth", 0.2123))))
    return bl


def matrad_dij(cubeRho, cubeMatIx, mcGeo, mcSrc, mcOpt, nargout=1):
    """[D, V] = omc_matrad(cubeRho, cubeMatIx, mcGeo, mcSrc, mcOpt)
    (omc_matrad.c:1417-1789).  Returns D, or (D, V) for nargout=2, as
    scipy.sparse.csc_matrix of shape (nx*ny*nz, nBixels)."""
    import scipy.sparse as sp
    if nargout > 2:
        raise MexError("matRad:matRad_ompInterface:invalidNumOutputs", "Too many output arguments.")
    _check_inputs(cubeRho, cubeMatIx, mcGeo, mcSrc)
    cube = _geometry(cubeRho, cubeMatIx, mcGeo)
    nsplit = int(_scalar(_field(mcOpt, "nSplit", required=True)))
    if not 1 <= nsplit <= 64:
        raise MexError("matRad:omc_matrad:Error", "nSplit must be between 1 and 64")
    ecut = _scalar(_field(mcOpt, "global_ecut", required=True))
    pcut = _scalar(_field(mcOpt, "global_pcut", required=True))
    seeds = np.asarray(_field(mcOpt, "randomSeeds", required=True), dtype=np.float64).ravel()
    seed = (int(seeds[0]) << 32) | (int(seeds[1]) if seeds.size > 1 else 0)
    files = [_field(mcOpt, k, required=True) for k in ("pegsFile", "pgs4formFile", "dataFolder")]
    _field(mcOpt, "outputFolder", required=True)
    nhist = int(_scalar(_field(mcOpt, "nHistories", 1e4)))
    nbatch = int(_scalar(_field(mcOpt, "nBatches", 10)))
    rel = _scalar(_field(mcOpt, "relDoseThreshold", 0.01))
    mode = {"event": EVENT_FP32, "plain": PLAIN_FP64}[str(_field(mcOpt, "transport", "event"))]
    device = int(_scalar(_field(mcOpt, "gpuDevice", 0)))
    bl = _source(mcSrc, mcOpt, cube)
    tables = _tables_for(files[0], files[1], files[2], cube.media)
    eng = Engine(tables, cube, ecut=ecut, pcut=pcut, device=device, nsplit=nsplit)
    try:
        colptr, rows, vals, var, _ = eng.run_beamlets(bl, nhist, nbatch, rel, seed=seed, mode=mode,
                                                      with_variance=nargout >= 2)
    finally:
        eng.close()
    shape = (int(np.prod(cube.shape)), len(bl["corner"]))
    D = sp.csc_matrix((vals, rows, colptr), shape=shape)
    if nargout < 2:
        return D
    return D, sp.csc_matrix((var, rows.copy(), colptr.copy()), shape=shape)
