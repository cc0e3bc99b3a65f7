"""Serving: continuous batching of beamlet and beam requests.

* isolation: a request's result is the same alone and in a mix of other
  requests admitted at different times (same request seed; only the FP64
  summation order of the tally atomics may differ, rtol 1e-9);
* the drain (the last particles run to the end in one launch once every
  admitted history is injected) changes no result: the same request with
  the drain off gives the same column;
* submissions from two producer threads while a third steps the server;
* admission by memory: with a budget for two requests, eight requests all
  finish, first come first served, with results identical to an unbounded
  server;
* a budget that holds no request fails with OMC_E_NOMEM;
* beam requests return the dense dose and uncertainty; latencies are
  reported per request."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bixels(engine_for):
    from ompmc_b200.engine import bixel_grid
    from tests.conftest import case_phantom
    ph = case_phantom("ctsmall")
    return bixel_grid(ph, [0.0, 51.0, 103.0, 154.0], bixel=1.0, field=(2.0, 2.0))


def run_all(server, reqs, budget_cycles=8):
    while server.step(budget_cycles) > 0:
        pass
    out = {}
    for name, rid in reqs.items():
        assert server.poll(rid) is not None
        out[name] = server.result_sparse(rid)
    return out


def test_result_same_alone_and_in_mix(engine_for, assets_root):
    from ompmc_b200.engine import Server, load_spectrum
    eng = engine_for("ctsmall")
    bl = bixels(engine_for)
    bl["spectrum"] = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    alone = Server(eng, seed=5)
    bs = alone.beamlet_set(bl)
    a = run_all(alone, {"x": alone.submit_beamlet(bs, 3, 30000, 10, 1e-4, seed=777)})["x"]
    alone.close()
    mix = Server(eng, seed=9)
    bs2 = mix.beamlet_set(bl)
    ids = {}
    for k in range(6):
        ids[f"pre{k}"] = mix.submit_beamlet(bs2, (k * 5) % 16, 20000 + 7000 * k, 10, 1e-4)
    mix.step(4)                                   # others already in flight
    ids["x"] = mix.submit_beamlet(bs2, 3, 30000, 10, 1e-4, seed=777)
    for k in range(4):
        ids[f"post{k}"] = mix.submit_beamlet(bs2, (k * 3 + 1) % 16, 15000, 10, 1e-4)
    res = run_all(mix, ids)
    b = res["x"]
    mix.close()
    assert np.array_equal(a[0], b[0])
    np.testing.assert_allclose(b[1], a[1], rtol=1e-9)
    np.testing.assert_allclose(b[2], a[2], rtol=1e-6, atol=1e-40)
    assert len(a[0]) > 100


def test_drain_changes_no_result(engine_for, assets_root):
    from ompmc_b200.engine import Server, load_spectrum
    eng = engine_for("ctsmall")
    bl = bixels(engine_for)
    bl["spectrum"] = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    out = []
    try:
        for drain in (0, -1):                     # default threshold, then off
            eng.event_params(drain_particles=drain)
            srv = Server(eng, seed=5)
            bs = srv.beamlet_set(bl)
            out.append(run_all(srv, {"x": srv.submit_beamlet(bs, 6, 40000, 10, 1e-4, seed=4242)})["x"])
            srv.close()
    finally:
        eng.event_params(drain_particles=0)
    a, b = out
    assert len(a[0]) > 100
    assert np.array_equal(a[0], b[0])
    np.testing.assert_allclose(b[1], a[1], rtol=1e-9)
    np.testing.assert_allclose(b[2], a[2], rtol=1e-6, atol=1e-40)


def test_admission_by_memory_budget(engine_for, assets_root):
    from ompmc_b200.engine import Server, load_spectrum
    eng = engine_for("ctsmall")
    bl = bixels(engine_for)
    bl["spectrum"] = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    nvox = int(np.prod(eng.shape))
    per_req = 10 * nvox * 8
    results = []
    for budget in (2 * per_req + 100, 0):
        s = Server(eng, mem_budget=budget, seed=3)
        bs = s.beamlet_set(bl)
        ids = {i: s.submit_beamlet(bs, i, 10000, 10, 1e-4, seed=100 + i) for i in range(8)}
        res = run_all(s, ids)
        lat = [s.poll(r) for r in ids.values()]
        assert all(l is not None and l > 0 for l in lat)
        results.append(res)
        s.close()
    for i in range(8):
        assert np.array_equal(results[0][i][0], results[1][i][0])
        np.testing.assert_allclose(results[0][i][1], results[1][i][1], rtol=1e-9)


def test_budget_too_small_is_nomem(engine_for):
    from ompmc_b200.engine import OmcError, Server
    eng = engine_for("ctsmall")
    with pytest.raises(OmcError) as ei:
        Server(eng, mem_budget=1000)
    assert ei.value.status == -11


def test_beam_request_matches_run_beam_statistically(engine_for, assets_root):
    from ompmc_b200.engine import EVENT_FP32, Server, load_spectrum
    from tests.conftest import CASES
    eng = engine_for("water30")
    spec = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    coll = CASES["water30"]["collimator"]
    s = Server(eng, seed=11)
    rid = s.submit_beam(400000, 10, spectrum=spec, collimator=coll, seed=99)
    while s.step(8) > 0:
        pass
    d1, u1 = s.result_dense(rid)
    s.close()
    d0, u0, _ = eng.run_beam(400000, 10, seed=5, mode=EVENT_FP32, spectrum=spec, collimator=coll)
    m = d0 > 0.2 * d0.max()
    z = (d1[m] - d0[m]) / np.sqrt((u1[m] * d1[m]) ** 2 + (u0[m] * d0[m]) ** 2)
    assert np.mean(np.abs(z) < 3) >= 0.99
    assert abs(z.mean()) < 0.25


def test_submissions_from_two_threads_while_a_third_steps(engine_for, assets_root):
    """Two producer threads submit beamlet requests while the main thread
    steps the server (omc_server_* serialise on the server's mutex).  Every
    request's column equals the one it gets submitted from one thread: a
    request's streams depend only on its seed, not on its id or timing."""
    import threading
    from ompmc_b200.engine import Server, load_spectrum
    eng = engine_for("ctsmall")
    bl = bixels(engine_for)
    bl["spectrum"] = load_spectrum(assets_root / "spectra" / "6mv.spectrum")
    jobs = [(i % 16, 8000 + 1000 * i, 500 + i) for i in range(12)]      # (bixel, histories, seed)
    one = Server(eng, seed=2)
    bs1 = one.beamlet_set(bl)
    ref = run_all(one, {k: one.submit_beamlet(bs1, b, n, 10, 1e-4, seed=sd) for k, (b, n, sd) in enumerate(jobs)})
    one.close()
    srv = Server(eng, seed=3)
    bs = srv.beamlet_set(bl)
    ids, errors = {}, []
    lock = threading.Lock()

    def produce(part):
        try:
            for k in part:
                b, n, sd = jobs[k]
                rid = srv.submit_beamlet(bs, b, n, 10, 1e-4, seed=sd)
                with lock:
                    ids[k] = rid
        except Exception as ex:           # reported by the main thread
            errors.append(ex)

    threads = [threading.Thread(target=produce, args=(range(p, len(jobs), 2),)) for p in range(2)]
    for t in threads:
        t.start()
    while any(t.is_alive() for t in threads) or srv.step(4) > 0:
        srv.step(2)
    for t in threads:
        t.join()
    assert not errors, errors
    assert sorted(ids) == list(range(len(jobs)))
    assert len(set(ids.values())) == len(jobs)
    got = run_all(srv, ids)
    srv.close()
    for k in range(len(jobs)):
        assert np.array_equal(got[k][0], ref[k][0])
        np.testing.assert_allclose(got[k][1], ref[k][1], rtol=1e-9)
