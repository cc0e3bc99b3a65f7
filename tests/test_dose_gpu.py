"""Statistical dose parity with the reference CPU code (omc_dosxyz CLI,
2e6 histories in 50 batches, tests/golden/dose_*.npz): in voxels above 10 %
of the reference maximum, z = (D_gpu - D_ref) / sqrt(s_gpu^2 + s_ref^2) with
s the batch-method standard errors, |z| < 3 in >= 99 % of them and no
systematic bias (mean z within 0.25), for the plain FP64 and the event FP32
forms."""
import numpy as np
import pytest

from tests.conftest import CASES

pytestmark = pytest.mark.gpu


def zscores(case, mode, golden, engine_for, assets_root, ncase=2_000_000, nbatch=50, seed=12345):
    from ompmc_b200.engine import load_spectrum
    g = golden(f"dose_{case}")
    eng = engine_for(case)
    spec = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    dose, unc, st = eng.run_beam(ncase, nbatch, seed=seed, mode=mode, spectrum=spec,
                                 collimator=CASES[case]["collimator"])
    assert st["flags"] == 0
    d = dose.ravel()[g["idx"]]
    u = unc.ravel()[g["idx"]]
    sel = g["dose"] > 0.10 * g["dmax"]
    s = np.sqrt((u * d) ** 2 + (g["unc"] * g["dose"]) ** 2)
    z = (d - g["dose"])[sel] / s[sel]
    return z, st


@pytest.mark.parametrize("mode", [0, 1], ids=["plain_fp64", "event_fp32"])
@pytest.mark.parametrize("case", ["water30", "slab64"])
def test_dose_z_scores(case, mode, golden, engine_for, assets_root):
    z, st = zscores(case, mode, golden, engine_for, assets_root)
    assert len(z) > 500
    frac = np.mean(np.abs(z) < 3)
    assert frac >= 0.99, f"{case} mode {mode}: |z|<3 in {frac:.4f}; mean z {z.mean():.3f}"
    assert abs(z.mean()) < 0.25, f"{case} mode {mode}: biased, mean z {z.mean():.3f}"
