"""Profiling of the event form: omc_profile_last, omc_profile_trace and
omc_profile_drain on a profiled slab run.

* the per-cycle trace injects every history once and its kernel times are
  positive; the per-kernel profile counts at least one electron launch per
  cycle;
* the drain record is the trace's last row (same device ms, same
  particles, at most the drain threshold) and its largest sub-history is
  consistent (events of the first particle <= events; steps >= 1);
* with the drain off the record is zeros, the trace has no drain row, and
  the dose is the same (the drain changes no trajectory; FP64 summation
  order only, rtol 1e-9)."""
import numpy as np
import pytest

from tests.conftest import CASES

pytestmark = pytest.mark.gpu

N = 300_000


def _run(eng, spec, **params):
    from ompmc_b200.engine import EVENT_FP32
    eng.event_params(**params)
    return eng.run_beam(N, 10, seed=11, mode=EVENT_FP32, spectrum=spec, collimator=CASES["slab64"]["collimator"])


def test_trace_and_drain_record(engine_for, assets_root):
    from ompmc_b200.engine import load_spectrum
    eng = engine_for("slab64", profile=True)
    spec = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    try:
        d1, _, st1 = _run(eng, spec, drain_particles=20000)
        tr = eng.profile_trace()
        dr = eng.profile_drain()
        pl = eng.profile_last()
        assert st1["flags"] == 0
        assert int(tr[:, 0].sum()) == N
        last = tr[-1]
        assert last[3] == 0 and last[4] == 0 and last[5] > 0          # the drain row
        assert (tr[:-1, 3:] > 0).any(axis=1).all()
        assert pl["electron"]["launches"] >= len(tr) - 1 > 0
        assert dr["ms"] == pytest.approx(last[5])
        assert dr["particles"] == int(last[1] + last[2])
        assert 0 < dr["particles"] <= 20000
        assert dr["max_events"] >= dr["max_chain_events"] >= 1
        assert dr["max_steps"] >= 1

        d2, _, st2 = _run(eng, spec, drain_particles=-1)
        tr2 = eng.profile_trace()
        dr2 = eng.profile_drain()
        assert st2["flags"] == 0
        assert dr2 == {"ms": 0.0, "particles": 0, "max_events": 0, "max_chain_events": 0, "max_steps": 0}
        assert not (tr2[-1, 3] == 0 and tr2[-1, 4] == 0)
        np.testing.assert_allclose(d2, d1, rtol=1e-9, atol=1e-30)
    finally:
        eng.event_params(drain_particles=0)
