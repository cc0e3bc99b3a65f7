"""Dose accuracy of the transport forms against a high-history FP64 oracle:
the heterogeneous slab workload (64^3 x 0.25 cm water / lung / bone /
water, 5x5 cm^2 6 MV-like) or the large CT-like phantom (256x256x160 x
0.2 cm, 10x10 cm^2 18 MV-like); ECUT 0.7 MeV, PCUT 0.01 MeV.

    python -m ompmc_b200.accuracy [--workload slab64|ct256-18mv] [--oracle-form plain|event64]
                                  [--oracle-hist 1e9] [--hist 1e7] [--plain-hist N] [--json out.json]

The oracle is an FP64 form at `--oracle-hist` histories: the plain form
(history-based, whose trajectories replay the reference's bit for bit) or
the FP64 event form (the same physics in FP64 with the event form's
transport; fast enough for 10^9 histories on the large phantom).  Each form
is then run at `--hist` histories (the plain form at `--plain-hist`), and
the FP32 event form again at the oracle's history count, so that a
systematic FP32 error would show above the noise.  For each run the table gives, in voxels above
50 % of the oracle maximum: the mean and maximum |D - D_oracle| / D_max, the
mean z = (D - D_oracle) / sigma (bias) and its spread, the fraction with
|z| < 3, and the gamma 2 %/2 mm pass rate against the oracle in voxels above
10 % of its maximum.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def _run(eng, n, mode, spec, coll, seed):
    t = time.perf_counter()
    d, u, st = eng.run_beam(int(n), 10, seed=seed, mode=mode, spectrum=spec, collimator=coll)
    return d, u, st, time.perf_counter() - t


def compare(d, u, d0, u0, bounds):
    from .gamma import gamma_pass_rate
    dmax = d0.max()
    m = d0 > 0.5 * dmax
    diff = (d - d0)[m]
    sig = np.sqrt((u * d) ** 2 + (u0 * d0) ** 2)[m]
    z = diff / np.where(sig > 0, sig, np.inf)
    idx = np.flatnonzero(d0.ravel() > 0.1 * dmax)
    rate, _ = gamma_pass_rate(idx, d0.ravel()[idx], d, bounds, dd=0.02, dta=0.2, cutoff=0.1, d_norm=dmax)
    return {"mean_abs_err_of_dmax": float(np.mean(np.abs(diff)) / dmax),
            "max_abs_err_of_dmax": float(np.max(np.abs(diff)) / dmax),
            "mean_z": float(np.mean(z)), "std_z": float(np.std(z)), "frac_abs_z_lt_3": float(np.mean(np.abs(z) < 3)),
            "gamma_2pct_2mm_pass": rate, "voxels_gt50": int(m.sum())}


WORKLOADS = {
    # name: (description, phantom, media, spectrum, collimator)
    "slab64": ("slab64 64^3 x 0.25 cm water/lung/bone/water, 5x5 cm2 6MV-like",
               lambda A: A.slab_phantom(64, 0.25), ["H2O521ICRU", "LUNG521ICRU", "ICRPBONE521ICRU"], "6mv",
               (-2.5, 2.5, -2.5, 2.5)),
    "ct256-18mv": ("ct256 256x256x160 x 0.2 cm CT-like (10.5 M voxels), 10x10 cm2 18MV-like",
                   lambda A: A.ct_phantom_large(), None, "18mv", (-5.0, 5.0, -5.0, 5.0)),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="slab64", choices=sorted(WORKLOADS))
    ap.add_argument("--oracle-form", default="plain", choices=["plain", "event64"],
                    help="FP64 oracle: the history-based plain form or the FP64 event form")
    ap.add_argument("--oracle-hist", type=float, default=1e9)
    ap.add_argument("--hist", type=float, default=1e7)
    ap.add_argument("--plain-hist", type=float, default=None, help="histories of the plain FP64 row (default --hist)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    from . import assets as A
    from .engine import EVENT_FP32, EVENT_FP64, PLAIN_FP64, Engine, Tables, load_spectrum
    root = A.require_assets()
    desc, mk, media, spec_name, coll = WORKLOADS[a.workload]
    ph = mk(A)
    spec = load_spectrum(root / "spectra" / f"{spec_name}.spectrum")
    eng = Engine(Tables.from_assets(media or A.CT_MEDIA, root), ph, device=a.device)
    bounds = (ph.xb, ph.yb, ph.zb)
    omode = PLAIN_FP64 if a.oracle_form == "plain" else EVENT_FP64
    d0, u0, st0, w0 = _run(eng, a.oracle_hist, omode, spec, coll, seed=1)
    out = {"workload": desc,
           "oracle": {"form": "plain FP64" if omode == PLAIN_FP64 else "event FP64", "histories": a.oracle_hist,
                      "seconds": w0, "mean_rel_unc_gt50": float(np.mean(u0[d0 > 0.5 * d0.max()]))},
           "runs": []}
    rows = (("plain FP64", PLAIN_FP64, a.plain_hist or a.hist), ("event FP64", EVENT_FP64, a.hist),
            ("event FP32/FP64 tally", EVENT_FP32, a.hist), ("event FP32/FP64 tally", EVENT_FP32, a.oracle_hist))
    for name, mode, n in rows:
        d, u, st, w = _run(eng, n, mode, spec, coll, seed=7)
        r = {"form": name, "histories": n, "seconds": w, "hist_per_s": n / st["seconds"]}
        r.update(compare(d, u, d0, u0, bounds))
        out["runs"].append(r)
        print(json.dumps(r), flush=True)
    eng.close()
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
