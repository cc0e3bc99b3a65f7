"""matRad MEX mirror (ompmc_b200.matrad.matrad_dij, omc_matrad.c:1417).

CPU: the argument checks raise the identifiers of the MEX entry's
mexErrMsgIdAndTxt calls (omc_matrad.c:157-175, 375-380) before any device
work.  GPU: D and V from the mirror agree with the unmodified MEX entry's
fixture (tests/golden/dij_ctsmall.npz) within statistics, with the row
numbering of a MATLAB column-major cube."""
import numpy as np
import pytest


def mex_inputs(assets_root, golden, nhist=None, fixture="dij_ctsmall"):
    from tests.conftest import case_phantom
    ph = case_phantom("ctsmall")
    g = golden(fixture)
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
    if int(g.get("gaussian", 0)):
        mcOpt.update(sourceGeometry="gaussian", sourceGaussianWidth=0.2123)
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
@pytest.mark.parametrize("fixture", ["dij_ctsmall", "dijg_ctsmall"], ids=["point", "gaussian"])
def test_mirror_matches_matrad_reference(fixture, transport, assets_root, golden):
    """dijg: the Gaussian focal spot (omc_matrad.c:1252-1295)."""
    from ompmc_b200.matrad import matrad_dij
    g = golden(fixture)
    args = mex_inputs(assets_root, golden, fixture=fixture)
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


# ------------------------------------------------ the C MEX entry
# ompmc_b200/mex/omc_matrad_gpu.c is what a MATLAB user compiles with `mex`;
# here it is compiled against the mex.h stand-in of the oracle and driven by
# the same harness that runs the unmodified reference entry.

def build_mex_shim(tmp_dir):
    """Shared library of the shim harness linked with omc_matrad_gpu.c."""
    import subprocess
    from tests.conftest import REPO
    shim = REPO / "oracle" / "mexshim"
    out = tmp_dir / "libomc_matrad_gpu_shim.so"
    steps = [["gcc", "-O2", "-fPIC", "-std=c99", "-Wall", "-Wextra", "-Werror", f"-I{shim}", f"-I{REPO / 'include'}",
              "-c", str(REPO / "ompmc_b200" / "mex" / "omc_matrad_gpu.c"), "-o", str(tmp_dir / "mex.o")],
             ["gcc", "-O2", "-fPIC", "-w", f"-I{shim}", "-c", str(shim / "harness_matrad.c"),
              "-o", str(tmp_dir / "shim.o")],
             ["gcc", "-shared", str(tmp_dir / "mex.o"), str(tmp_dir / "shim.o"), f"-L{REPO / 'ompmc_b200'}",
              "-lomcgpu", f"-Wl,-rpath,{REPO / 'ompmc_b200'}", "-lm", "-o", str(out)]]
    for cmd in steps:
        p = subprocess.run(cmd, capture_output=True, text=True)
        assert p.returncode == 0, p.stderr[-2000:]
    return out


def test_mex_entry_builds_against_mex_api(tmp_path):
    """The MEX source compiles warning-free against the mx/mex API subset
    and exports mexFunction (no device needed)."""
    import ctypes
    lib = ctypes.CDLL(str(build_mex_shim(tmp_path)))
    assert hasattr(lib, "mexFunction") and hasattr(lib, "hm_dij")


@pytest.mark.gpu
def test_mex_entry_matches_matrad_reference(tmp_path, assets_root, golden):
    """D and V of the C MEX entry (event form, the default) against the
    unmodified reference entry's fixture, as for the Python mirror."""
    from oracle.ref import matrad_dij as shim_dij
    from tests.conftest import case_phantom
    g = golden("dij_ctsmall")
    lib = build_mex_shim(tmp_path)
    ph = case_phantom("ctsmall")
    bl = dict(src=g["src"], corner=g["corner"], side1=g["side1"], side2=g["side2"], ibeam=g["ibeam"])
    colptr, rows, vals, var = shim_dij(ph, bl, int(g["nhist"]), int(g["nbatch"]), seeds=(97, 33),
                                       rel_threshold=float(g["rel"]),
                                       spectrum_file=str(assets_root / "spectra" / "6mv.spectrum"), lib=lib)
    nvox = int(np.prod(ph.shape))
    zs = []
    for i in range(len(g["corner"])):
        rr = g["rows"][g["colptr"][i]:g["colptr"][i + 1]]
        rv = g["vals"][g["colptr"][i]:g["colptr"][i + 1]]
        rvar = g["var"][g["colptr"][i]:g["colptr"][i + 1]]
        col = np.zeros(nvox)
        vcol = np.zeros(nvox)
        col[rows[colptr[i]:colptr[i + 1]]] = vals[colptr[i]:colptr[i + 1]]
        vcol[rows[colptr[i]:colptr[i + 1]]] = var[colptr[i]:colptr[i + 1]]
        sel = rv > 0.05 * rv.max()
        zs.append((col[rr[sel]] - rv[sel]) / np.sqrt(vcol[rr[sel]] + rvar[sel]))
    z = np.concatenate(zs)
    assert len(z) > 250
    assert np.mean(np.abs(z) < 3) >= 0.99, np.mean(np.abs(z) < 3)
    assert abs(z.mean()) < 0.25
