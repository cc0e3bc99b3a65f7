"""Autotuner (ompmc_b200.autotune): the search returns a setting from its
space, leaves the engine at it, and the tuned engine's dose equals the
default engine's (at the same electron_chsteps) up to the FP64 summation
order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tune_beam_small_space(engine_for, assets_root):
    from ompmc_b200.autotune import tune_beam
    from ompmc_b200.engine import EVENT_FP32, Engine, Tables, load_spectrum
    from tests.conftest import CASES, case_phantom
    spec = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    coll = CASES["slab64"]["collimator"]
    t = Tables.from_assets(CASES["slab64"]["media"], assets_root)
    ph = case_phantom("slab64")
    eng = Engine(t, ph)
    from ompmc_b200.engine import OmcError
    with pytest.raises(OmcError):
        eng.event_params(block=512)            # above the transport kernels' launch bound
    with pytest.raises(OmcError):
        eng.event_params(block=100)            # not whole warps
    space = {"electron_tsteps": [1, 2], "tail_boost": [1, 32], "inflight": [1 << 18, 1 << 20], "block": [128, 256]}
    cfg, rate, trials = tune_beam(eng, nhist=100_000, space=space, repeats=1, spectrum=spec, collimator=coll)
    assert all(cfg[k] in v for k, v in space.items())
    assert rate > 0 and len(trials) >= 5
    d1, _, _ = eng.run_beam(100_000, 10, seed=5, mode=EVENT_FP32, spectrum=spec, collimator=coll)
    eng.close()
    # electron_chsteps changes which random numbers a trajectory draws (not
    # the distribution it samples): the reference uses the tuned value
    ref = Engine(t, ph, electron_chsteps=cfg["electron_chsteps"])
    d0, _, _ = ref.run_beam(100_000, 10, seed=5, mode=EVENT_FP32, spectrum=spec, collimator=coll)
    ref.close()
    m = d0 > 0
    assert np.array_equal(d1 > 0, m)
    np.testing.assert_allclose(d1[m], d0[m], rtol=1e-9)
