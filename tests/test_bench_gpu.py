"""bench.py's GPU helpers on a few requests of the beamlet load: the
profiled pass the roofline line is built from (device counters of every
transport kernel) and requests served one at a time (the reference's
mode), whose columns must come back."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_profiled_pass_counters():
    import bench
    from ompmc_b200.workloads import beamlet_load
    load = beamlet_load(7)
    prof, hist, n = bench.profiled_pass(load, 0, 3, 4000.0, max_requests=3, queue_capacity=1 << 20)
    assert n == 3 and hist == float(np.sum(load["nhist"][:3]))
    ek, pk = prof["electron"], prof["photon"]
    assert ek["launches"] > 0 and ek["seconds"] > 0 and pk["seconds"] > 0
    # every history starts as a photon; electrons take several condensed-
    # history steps per event and deposit several times per history
    assert pk["particles"] >= hist
    assert ek["particles"] > 0 and ek["steps"] >= ek["particles"]
    assert ek["dep"] > hist and 0 < ek["atom"] <= ek["dep"]


def test_requests_one_at_a_time():
    import bench
    from ompmc_b200.engine import Server
    from ompmc_b200.workloads import beamlet_load
    load = beamlet_load(7)
    eng = bench.beamlet_engine(load, 0)
    srv = Server(eng, seed=3)
    lat, rate = bench.serve_sequential(srv, load, 3, 11)
    srv.close()
    eng.close()
    assert lat.shape == (3,) and np.all(lat > 0)
    assert rate > 0
