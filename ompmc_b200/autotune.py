"""Autotuner of the event form's launch parameters.

The event form's results do not depend on its tuning parameters (particle
streams are keyed by history and stream position, so only the FP64
summation order of the tallies changes), which leaves them free to be picked
for speed per phantom, source and GPU:

* electron_tsteps — tstep-loop iterations per electron event while the
  queues fill the GPU;
* tail_boost      — how far that budget may grow as the queues drain;
* inflight        — particles kept in the queues by the injector;
* block           — threads per block of the transport kernels (whole warps,
                    at most 256, their launch bound);
* electron_split  — regroup energy: electrons above it (kinetic, MeV) are
                    queued apart from the others (0 = one group);
* electron_chsteps — condensed-history steps between re-draws of an
                    electron's distance to its next discrete interaction;
* drain_particles — particles left at which the run switches from cycles
                    to the drain kernel (-1 never, 0 default).

`tune_beam` runs short dose runs of the given beam on a live engine and
searches the space coordinate by coordinate (each parameter swept with the
others at their best so far, twice over), keeping the fastest; the engine is
left at the best setting.  `load`/`save` keep results in a JSON file keyed
by GPU, phantom shape, media and source.
"""
from __future__ import annotations

import json
import time
from pathlib import Path

SPACE = {
    "electron_tsteps": [1, 2, 3, 4, 6],
    "tail_boost": [1, 8, 32, 128],
    "inflight": [1 << 18, 1 << 19, 1 << 20, 1 << 21],
    "block": [64, 128, 256],
    "electron_split": [0.0, 0.1, 0.15, 0.2, 0.3, 0.5, 1.0],
    "electron_chsteps": [1, 2, 3, 4, 8],
    "drain_particles": [-1, 10000, 20000, 40000, 80000],
}
# the starting point: the best setting measured on the slab workload
DEFAULT = {"electron_tsteps": 1, "tail_boost": 32, "inflight": 1 << 21, "block": 256, "electron_split": 0.0,
           "electron_chsteps": 3, "drain_particles": 40000}


def _rate(eng, cfg, nhist, run_kw, repeats):
    from .engine import EVENT_FP32
    eng.event_params(**cfg)
    eng.run_beam(max(nhist // 8, 1000), 10, seed=11, mode=EVENT_FP32, **run_kw)
    best = float("inf")
    for r in range(repeats):
        _, _, st = eng.run_beam(nhist, 10, seed=12 + r, mode=EVENT_FP32, **run_kw)
        best = min(best, st["seconds"])
    return nhist / best


def tune_beam(eng, nhist=200_000, space=None, repeats=2, rounds=2, log=None, **run_kw):
    """Coordinate search over `space` (default SPACE) with dose runs of
    `nhist` histories of the beam given by `run_kw` (spectrum, collimator,
    ...).  Returns (best config, histories/s, list of (config, rate))."""
    space = dict(space or SPACE)
    # start from DEFAULT, each parameter moved into the searched values
    cur = {k: (v if k not in space or v in space[k] else space[k][0]) for k, v in DEFAULT.items()}
    seen = {}

    def measure(cfg):
        key = tuple(sorted(cfg.items()))
        if key not in seen:
            t = time.perf_counter()
            seen[key] = _rate(eng, cfg, nhist, run_kw, repeats)
            if log:
                log(f"{cfg} -> {seen[key] / 1e6:.2f} M hist/s ({time.perf_counter() - t:.1f} s)")
        return seen[key]

    best_rate = measure(cur)
    for _ in range(rounds):
        changed = False
        for name, values in space.items():
            for v in values:
                cfg = dict(cur, **{name: v})
                r = measure(cfg)
                # a change must beat the best so far by more than the
                # run-to-run spread of the short runs (about 1 %)
                if r > best_rate * 1.02:
                    best_rate, cur, changed = r, cfg, True
        if not changed:
            break
    eng.event_params(**cur)
    trials = [(dict(k), r) for k, r in seen.items()]
    return cur, best_rate, trials


def cache_key(gpu_name, phantom, media, source):
    return f"{gpu_name}|{'x'.join(str(n) for n in phantom.shape)}|{','.join(media)}|{source}"


def load(path, key):
    p = Path(path)
    if not p.exists():
        return None
    return json.loads(p.read_text()).get(key)


def save(path, key, cfg, rate):
    p = Path(path)
    data = json.loads(p.read_text()) if p.exists() else {}
    data[key] = dict(cfg, hist_per_s=rate)
    p.write_text(json.dumps(data, indent=1, sort_keys=True))
