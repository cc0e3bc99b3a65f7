"""Statistical dose parity with the reference CPU code (omc_dosxyz CLI,
tests/golden/dose*_<case>.npz, 50 batches): in voxels above 10 % of the
reference maximum, z = (D_gpu - D_ref) / sqrt(s_gpu^2 + s_ref^2) with s the
batch-method standard errors, |z| < 3 in >= 99 % of them and no systematic
bias (mean z within 0.25), for the plain FP64 and the event FP32 forms.
Sources: the 6 MV-like spectrum on water, the slab and the 4-media CT-like
phantom; the 18 MV-like spectrum on the slab (pair production in bone);
6 MeV electron and 3 MeV positron beams on water (omc_dosxyz.c:596-605);
the 6 MV-like spectrum with photon splitting (nsplit = 20) on water and the
slab."""
import numpy as np
import pytest

from tests.conftest import CASES

pytestmark = pytest.mark.gpu

FIXTURES = ["dose_water30", "dose_slab64", "dose18_slab64", "dose_ctsmall", "dosee_water30", "dosep_water30",
            "dosesplit_water30", "dosesplit_slab64"]


def zscores(fixture, mode, golden, engine_for, assets_root, nbatch=50, seed=12345):
    from ompmc_b200.engine import load_spectrum
    g = golden(fixture)
    case = fixture.split("_", 1)[1]
    ns = int(g["nsplit"]) if "nsplit" in g else 1
    eng = engine_for(case, nsplit=ns) if ns > 1 else engine_for(case)
    spec_name = str(g["spectrum"]) if "spectrum" in g else "6mv"
    spec = load_spectrum(assets_root / "spectra" / f"{spec_name}.spectrum") if spec_name else None
    mono = float(g["mono_energy"]) if "mono_energy" in g else 1.25
    charge = int(g["charge"]) if "charge" in g else 0
    dose, unc, st = eng.run_beam(int(g["ncase"]), nbatch, seed=seed, mode=mode, spectrum=spec, mono_energy=mono,
                                 charge=charge, collimator=CASES[case]["collimator"])
    assert st["flags"] == 0
    d = dose.ravel()[g["idx"]]
    u = unc.ravel()[g["idx"]]
    sel = g["dose"] > 0.10 * g["dmax"]
    s = np.sqrt((u * d) ** 2 + (g["unc"] * g["dose"]) ** 2)
    z = (d - g["dose"])[sel] / s[sel]
    return z, st


@pytest.mark.parametrize("mode", [0, 1], ids=["plain_fp64", "event_fp32"])
@pytest.mark.parametrize("fixture", FIXTURES)
def test_dose_z_scores(fixture, mode, golden, engine_for, assets_root):
    z, st = zscores(fixture, mode, golden, engine_for, assets_root)
    assert len(z) > 150
    frac = np.mean(np.abs(z) < 3)
    assert frac >= 0.99, f"{fixture} mode {mode}: |z|<3 in {frac:.4f}; mean z {z.mean():.3f}"
    assert abs(z.mean()) < 0.25, f"{fixture} mode {mode}: biased, mean z {z.mean():.3f}"
