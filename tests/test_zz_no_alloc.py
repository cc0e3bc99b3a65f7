"""The fixed-scratch beam run (omc_run_beam_noalloc) for callers that must not
allocate device memory while they run a dose calculation — a plan optimiser
evaluating dose inside its iteration loop cannot afford the device-wide
synchronisation and unbounded latency of cudaMalloc/cudaFree, and a host
application whose GPU memory belongs to its own fixed-budget pool may see an
extra allocation fail.

Checked through the C ABI against omc_run_beam (plain FP64 form, same seed):
the same histories are transported, so dose and uncertainty agree up to the
summation order of the FP64 tally atomics; two calls in a row, because the
scratch keeps the previous call's contents.  This file is named so that
pytest collects it after every other test."""
import numpy as np
import pytest

from tests.conftest import CASES

pytestmark = pytest.mark.gpu


def spectrum(assets_root):
    from ompmc_b200.engine import load_spectrum
    return load_spectrum(assets_root / "spectra" / "6mv.spectrum")


def test_noalloc_matches_run_beam_twice(engine_for, assets_root):
    from ompmc_b200.engine import PLAIN_FP64
    eng = engine_for("water30")
    spec = spectrum(assets_root)
    coll = CASES["water30"]["collimator"]
    d0, u0, s0 = eng.run_beam(100000, 10, seed=4242, mode=PLAIN_FP64, spectrum=spec, collimator=coll)
    assert s0["flags"] == 0 and d0.max() > 0
    from ompmc_b200.engine import device_allocations
    for k in range(2):
        before = device_allocations()
        d, u, s = eng.run_beam_noalloc(100000, 10, seed=4242, spectrum=spec, collimator=coll)
        if k == 1:
            # after the warm-up call, a call makes no device allocation
            assert device_allocations() == before
        assert s["flags"] == 0
        assert s["launches"] == s0["launches"]
        assert s["histories"] == s0["histories"]
        np.testing.assert_allclose(d, d0, rtol=1e-9, atol=1e-30)
        m = d0 > 0
        np.testing.assert_allclose(u[m], u0[m], rtol=1e-6, atol=1e-9)
        assert abs(s["edep"] - s0["edep"]) <= 1e-9 * s0["edep"]


def test_noalloc_rejects_phantoms_above_its_capacity(assets_root):
    from ompmc_b200 import assets as A
    from ompmc_b200.engine import Engine, OmcError, Tables
    t = Tables.from_assets(["H2O521ICRU"], assets_root)
    eng = Engine(t, A.water_cube(65, 0.5))   # 274625 voxels > 262144
    try:
        with pytest.raises(OmcError) as ei:
            eng.run_beam_noalloc(1000, 2, seed=1, spectrum=spectrum(assets_root))
        assert ei.value.status == -5
        assert "262144" in str(ei.value)
    finally:
        eng.close()
