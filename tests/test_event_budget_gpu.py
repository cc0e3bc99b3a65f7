"""Event budgets do not change results.

An event-form particle resumes its Philox stream at the exact position it
stopped at, secondaries are keyed by their parent's stream position at
creation, and FP32 directions are renormalised inside the physics, so where
a cycle cuts a particle's transport is invisible in its trajectory.  The
dose of a run with the smallest fixed budgets (one photon interaction, one
electron tstep-loop iteration per event) equals the dose with the adaptive
drain-tail budgets, with large fixed ones and with the electron queues
regrouped by energy, smaller blocks and fewer particles in flight, with the
interactions sampled in their own kernel and with the remaining particles
run to completion by the drain kernel at any point after the last
injection, up to the summation order of the FP64 tally atomics (rtol 1e-9
per voxel)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


CONFIGS = {
    "nsplit1": [dict(electron_tsteps=1, tail_boost=1, electron_split=0.0), dict(),
                dict(electron_tsteps=7, tail_boost=64), dict(electron_split=1.0, block=128, inflight=1 << 18),
                dict(electron_interact_kernel=1, electron_tsteps=3),
                # the drain: never, and as early as every history is in
                dict(drain_particles=-1), dict(drain_particles=1 << 22)],
    # photon splitting: a split photon's state (sub-photon, survivor,
    # stratification offset) is carried from event to event
    "nsplit5": [dict(nsplit=5, electron_tsteps=1, tail_boost=1, electron_split=0.0), dict(nsplit=5),
                dict(nsplit=5, block=128, inflight=1 << 18), dict(nsplit=5, drain_particles=-1),
                dict(nsplit=5, drain_particles=1 << 22)],
}


@pytest.mark.parametrize("split", ["nsplit1", "nsplit5"])
@pytest.mark.parametrize("case", ["slab64", "ctsmall"])
def test_dose_independent_of_event_budgets(case, split, assets_root):
    from ompmc_b200.engine import EVENT_FP32, Engine, Tables, load_spectrum
    from tests.conftest import CASES, case_phantom
    ph = case_phantom(case)
    t = Tables.from_assets(CASES[case]["media"], assets_root)
    spec = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    coll = CASES[case]["collimator"]
    doses = []
    for kw in CONFIGS[split]:
        eng = Engine(t, ph, **kw)
        d, u, st = eng.run_beam(200000 if split == "nsplit1" else 50000, 10, seed=4242, mode=EVENT_FP32, spectrum=spec, collimator=coll)
        assert st["flags"] == 0
        doses.append(d)
        eng.close()
    m = doses[0] > 0
    assert m.sum() > 1000
    for d in doses[1:]:
        assert np.array_equal(d > 0, m)
        np.testing.assert_allclose(d[m], doses[0][m], rtol=1e-9)
