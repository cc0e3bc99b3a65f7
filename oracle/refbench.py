"""CPU reference of the beamlet serving benchmark: the unmodified matRad D_ij
entry (ucodes/omc_matrad/omc_matrad.c:1417-1789), built with OpenMP by
oracle/Makefile into oracle/_ref/libompmc_matrad_omp.so and driven through
the mex.h shim.

Test infrastructure only: used by the reference arm and the CPU-baseline leg
of bench.py, never by the product.

The reference takes one history count per call (mcOpt.nHistories), while
every beamlet request of the load has its own, so each beamlet is one call.
A call initialises the tables, then runs its beamlet loop (batches in
parallel over the host cores, omc_matrad.c:1576-1720); the time of that
loop is read from the shim's record of the waitbar calls the entry makes
before and after it (oracle/mexshim/harness_matrad.c), so per-call
initialisation is not counted.  One beamlet per call also keeps the
variance output clean (the entry does not reset its sum of squares between
beamlets, omc_matrad.c:1702).

    python -m oracle.refbench --picks 3,17,40 --nhist 20000,51230,80000 [--seed 7]

prints one JSON object: per beamlet its bixel, histories, loop seconds and
the mean relative uncertainty of its column above 50 % of its maximum.
Run it under `taskset` to choose the cores (omp_get_num_procs follows the
affinity mask, omc_matrad.c:1449).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
OMP_LIB = HERE / "_ref" / "libompmc_matrad_omp.so"


def available():
    return OMP_LIB.exists()


def run(picks, nhist, seed=7):
    """Runs the beamlets `picks` of the load with `nhist` histories each, one
    reference call per beamlet, on the cores this process may use."""
    sys.path.insert(0, str(REPO))
    from oracle.ref import matrad_dij
    from ompmc_b200.workloads import LOAD_NBATCH, LOAD_REL, beamlet_load, column_unc
    load = beamlet_load(seed)
    ph, bl = load["phantom"], load["beamlets"]
    L = C.CDLL(str(OMP_LIB))
    L.hm_timing(1)
    L.hm_waitbar_log.restype = C.c_int
    tbuf = np.zeros(4096)
    pbuf = np.zeros(4096)
    out = []
    for k, (b, n) in enumerate(zip(picks, nhist)):
        one = dict(bl, corner=bl["corner"][b:b + 1], side1=bl["side1"][b:b + 1], side2=bl["side2"][b:b + 1],
                   ibeam=bl["ibeam"][b:b + 1])
        jc, ir, pr, var = matrad_dij(ph, one, int(n), LOAD_NBATCH, seeds=(97, 33 + k), rel_threshold=LOAD_REL,
                                     spectrum_file=str(load["spectrum_file"]), lib=OMP_LIB)
        m = L.hm_waitbar_log(tbuf.ctypes.data_as(C.POINTER(C.c_double)),
                             pbuf.ctypes.data_as(C.POINTER(C.c_double)), len(tbuf))
        if m < 2:
            raise RuntimeError("the reference made no waitbar calls: verbose timing not active")
        # first call: the waitbar is created before the loop; last: closed after it
        loop_s = float(tbuf[m - 1] - tbuf[0])
        out.append(dict(bixel=int(b), nhist=int(n), loop_s=loop_s, nnz=int(len(pr)), unc=column_unc(pr, var)))
    return out


def run_pinned(picks, nhist, cores, seed=7, timeout=3600):
    """`run` in a child process pinned to the first `cores` host cores."""
    cmd = [sys.executable, "-m", "oracle.refbench", "--picks", ",".join(str(int(p)) for p in picks),
           "--nhist", ",".join(str(int(n)) for n in nhist), "--seed", str(seed)]
    cmd = ["taskset", "-c", f"0-{cores - 1}"] + cmd
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, cwd=str(REPO),
                       env=dict(os.environ, PYTHONPATH=str(REPO)))
    if p.returncode != 0:
        raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
    return json.loads(p.stdout.strip().splitlines()[-1])["beamlets"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--picks", required=True)
    ap.add_argument("--nhist", required=True)
    ap.add_argument("--seed", type=int, default=7)
    a = ap.parse_args()
    picks = [int(x) for x in a.picks.split(",")]
    nhist = [int(x) for x in a.nhist.split(",")]
    res = run(picks, nhist, a.seed)
    print(json.dumps({"cores": len(os.sched_getaffinity(0)), "beamlets": res}))


if __name__ == "__main__":
    main()
