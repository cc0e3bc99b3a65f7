"""Gamma 2 %/2 mm of the FP32 event form against the reference CLI.

Reference: tests/golden/gamma_<case>.npz, the unmodified ompMC CLI at high
statistics (water30 1e8, slab64 4e8 histories).  The event form runs twice
the reference's histories so that its own noise is the smaller part.
Criterion (global, normalised to the reference maximum): gamma <= 1 in at
least 99 % of the voxels above 10 % of the maximum."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HIST = {"water30": 200_000_000, "slab64": 800_000_000}


@pytest.mark.parametrize("case", ["water30", "slab64"])
def test_gamma_event_form_vs_reference(case, golden, engine_for, assets_root):
    from ompmc_b200.engine import EVENT_FP32, load_spectrum
    from ompmc_b200.gamma import gamma_pass_rate
    from tests.conftest import CASES, case_phantom
    g = golden(f"gamma_{case}")
    ph = case_phantom(case)
    eng = engine_for(case)
    spec = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    d, u, st = eng.run_beam(HIST[case], 10, seed=31337, mode=EVENT_FP32, spectrum=spec,
                            collimator=CASES[case]["collimator"])
    assert st["flags"] == 0
    rate, gam = gamma_pass_rate(g["idx"], g["dose"], d, (ph.xb, ph.yb, ph.zb), dd=0.02, dta=0.2, cutoff=0.1,
                                d_norm=float(g["dmax"]))
    assert len(gam) > 1000
    assert rate >= 0.99, f"gamma 2%/2mm pass rate {rate:.4f}"
