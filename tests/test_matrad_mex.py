"""matRad MEX mirror (ompmc_b200.matrad.matrad_dij, omc_matrad.c:1417).

CPU: the argument checks raise the identifiers of the MEX entry's
mexErrMsgIdAndTxt calls (omc_matrad.c:157-175, 375-380) before any device
work.  GPU: D and V from the mirror agree with the unmodified MEX entry's
fixture (tests/golden/dij_ctsmall.npz) within statistics, with the row
numbering of a MATLAB column-major cube."""
import numpy as np
import pytest


def mex_inputs(assets_root, golden, nhist=None):
    from tests.conftest import case_phantom
    ph = case_phantom("ctsmall")
    g = golden("dij_ctsmall")
    cubeRho = np.ascontiguousarray(ph.rho.transpose(2, 1, 0))        # (nx, ny, nz) MATLAB indexing
    cubeMatIx = np.ascontiguousarray(ph.med.transpose(2, 1, 0)).astype(np.int32)
    mcGeo = dict(material=[[m, ""] for m in ph.media], xBounds=ph.xb, yBounds=ph.yb, zBounds=ph.zb)
    src, cor, s1, s2 = g["src"], g["corner"], g["side1"], g["side2"]
    mcSrc = dict(nBixels=len(cor), iBeam=g["ibeam"].astype(np.float64) + 1,
                 xSource=src[:, 0], ySource=src[:, 1], zSource=src[:, 2],
                 xCorner=cor[:, 0], yCorner=cor[:, 1], zCorner=cor[:, 2],
                 xSide1=s1[:, 0], ySide1=s1[:, 1], zSide1=s1[:, 2],
                 xSide2=s2[:, 0], ySide2=s2[:, 1], zSide2=s2[:, 2])
    mcOpt = dict(verbose=0, nHistories=int(nhist or g["nhist"]), nBatches=int(g["nbatch"]), nSplit=1,
                 spectrumFile=str(assets_root / "spectra" / "6mv.spectrum"), monoEnergy=0.1, charge=0,
                 global_ecut=0.7, global_pcut=0.01, randomSeeds=[97, 33],
                 pegsFile=str(assets_root / "pegs4" / "521icru.pegs4dat"),
                 pgs4formFile=str(assets_root / "pegs4" / "pgs4form.dat"),
                 dataFolder=str(assets_root / "data") + "/", outputFolder=str(assets_root / "out") + "/",
                 relDoseThreshold=float(g["rel"]))
    return cubeRho, cubeMatIx, mcGeo, mcSrc, mcOpt


@pytest.mark.parametrize("mutate,ident", [
    (lambda a: a.__setitem__(0, a[0].astype(np.float32)), "matRad:matRad_ompInterface:inputNotDouble"),
    (lambda a: a.__setitem__(0, a[0][:, :, 0]), "matRad:matRad_ompInterface:inputNot3D"),
    (lambda a: a.__setitem__(1, a[1].astype(np.int64)), "matRad:matRad_ompInterface:inputNotInt32"),
    (lambda a: a.__setitem__(2, [1, 2]), "MATLAB:phonebook:inputNotStruct"),
    (lambda a: a.__setitem__(3, None), "MATLAB:phonebook:inputNotStruct"),
    (lambda a: a[2].pop("material"), "matRad:omc_matrad:Error"),
    (lambda a: a[4].pop("global_ecut"), "matRad:omc_matrad:Error"),
    (lambda a: a[4].__setitem__("nSplit", 65), "matRad:omc_matrad:Error"),
    (lambda a: a[4].__setitem__("spectrumFile", "/nonexistent/x.spectrum"), "matRad:omc_matrad:Error"),
], ids=["rho_not_double", "rho_not_3d", "matix_not_int32", "geo_not_struct", "src_not_struct",
        "no_materials", "missing_ecut", "nsplit", "no_spectrum"])
def test_argument_checks(mutate, ident, assets_root, golden):
    from ompmc_b200.matrad import MexError, matrad_dij
    args = list(mex_inputs(assets_root, golden))
    mutate(args)
    with pytest.raises(MexError) as ei:
        matrad_dij(*args)
    assert ei.value.identifier == ident


def test_too_many_outputs(assets_root, golden):
    from ompmc_b200.matrad import MexError, matrad_dij
    with pytest.raises(MexError):
        matrad_dij(*mex_inputs(assets_root, golden), nargout=3)


@pytest.mark.gpu
@pytest.mark.parametrize("transport", ["event", "plain"])
def test_mirror_matches_matrad_reference(transport, assets_root, golden):
    from ompmc_b200.matrad import matrad_dij
    g = golden("dij_ctsmall")
    args = mex_inputs(assets_root, golden)
    args[4]["transport"] = transport
    D, V = matrad_dij(*args, nargout=2)
    nvox = int(np.prod(args[0].shape))
    assert D.shape == (nvox, len(g["corner"])) and V.shape == D.shape
    zs = []
    for i in range(D.shape[1]):
        rr = g["rows"][g["colptr"][i]:g["colptr"][i + 1]]
        rv = g["vals"][g["colptr"][i]:g["colptr"][i + 1]]
        rvar = g["var"][g["colptr"][i]:g["colptr"][i + 1]]
        col = D[:, i].toarray().ravel()
        vcol = V[:, i].toarray().ravel()
        sel = rv > 0.05 * rv.max()
        zs.append((col[rr[sel]] - rv[sel]) / np.sqrt(vcol[rr[sel]] + rvar[sel]))
    z = np.concatenate(zs)
    assert len(z) > 250
    assert np.mean(np.abs(z) < 3) >= 0.99, np.mean(np.abs(z) < 3)
    assert abs(z.mean()) < 0.25
