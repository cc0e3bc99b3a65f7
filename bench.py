"""Benchmark: the served beamlet dose-influence load on one B200, one JSON
line on stdout.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload beamlets|slab64]

Workload (default, `beamlets`): 2023 beamlet requests, the dose-influence
columns of a 7-beam coplanar plan (gantry 0, 51, 103, 154, 206, 257, 309
degrees; 17 x 17 bixels of 0.5 cm at the isocentre, SAD 100 cm) on the seeded
128x128x96 x 0.3 cm CT-like phantom, the 6 MV-like spectrum, histories per
request log-uniform in [2e4, 2e5] (1.58e8 in all), 10 batches, sparse columns
thresholded at 1e-4 of their maximum with the variance of the mean beside
them.  A step is one pass of the whole load through the continuous-batching
server (omc_server_*): requests arrive as a Poisson process (default
4000/s, above what one GPU serves, so the server works through a backlog
with every slot busy) and are admitted as slots and device memory free up;
each finished column is copied into host memory as it is reported.
`value` is the load's histories over the device time of the passes (CUDA
events on the server's stream); `e2e` is the same over host wall-clock
time, from the first submission to the last column in host memory.
p50_ms/p99_ms are per-beamlet latencies (arrival to column in host memory)
of one more pass at `--latency-load` of the measured throughput; the
saturated passes' latencies are reported beside them.  `unc` gives the mean
relative uncertainty of each column above 50 % of its maximum and the
seconds to 1 % it implies.

`--impl reference` runs ompMC's own matRad D_ij entry (omc_matrad.c,
unmodified, built with OpenMP into oracle/_ref) on all host cores, one call
per beamlet of a different sample of the same load each step, timing each
call's beamlet loop.

`--workload slab64` keeps the single-beam dose run: 10^7 histories of a 5x5
cm^2 6 MV-like beam on the 64^3 x 0.25 cm water/lung/bone slab phantom
through omc_run_beam per step.  Under torchrun every rank runs its own
histories on its own GPU (weak scaling, no collective on the data path); the
reported time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "histories/s at 1% dose unc. (served vs plain GPU vs CPU); p50/p99 beamlet ms"
WORKLOAD = ("beamlets: 2023 beamlet requests (7 coplanar beams x 17x17 bixels of 0.5 cm) on the 128x128x96 x 0.3 cm "
            "CT-like phantom, 6MV-like, log-uniform 2e4-2e5 histories, 10 batches, sparse columns at 1e-4, Poisson "
            "arrivals, served")
SLAB_WORKLOAD = ("slab64: 64^3 x 0.25 cm water/lung(0.26)/bone(1.85)/water, 5x5 cm2 6MV-like, 1e7 histories in 10 "
                 "batches per step")
HIST_PER_STEP = 10_000_000
NBATCH = 10
COLLIMATOR = (-2.5, 2.5, -2.5, 2.5)
MEDIA = ["H2O521ICRU", "LUNG521ICRU", "ICRPBONE521ICRU"]


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def workload_inputs():
    from ompmc_b200 import assets as A
    root = A.require_assets()
    ph = A.slab_phantom(64, 0.25)
    spec_path = root / "spectra" / "6mv.spectrum"
    if not spec_path.exists():
        A.write_spectrum(spec_path, "6mv")
    return root, ph, spec_path


def mean_unc_above_half(dose, unc):
    m = dose > 0.5 * dose.max()
    return float(unc[m].mean())


def atomic_peak(device, n_vox):
    """Measured FP64 scattered-add throughput (torch index_add_ on the GPU):
    the denominator for the tally-atomic fraction."""
    import torch
    dev = torch.device("cuda", device)
    tally = torch.zeros(n_vox, dtype=torch.float64, device=dev)
    n = 1 << 24
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    idx = torch.randint(0, n_vox, (n,), device=dev, generator=g)
    val = torch.rand(n, dtype=torch.float64, device=dev, generator=g)
    for _ in range(3):
        tally.index_add_(0, idx, val)
    torch.cuda.synchronize(dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    reps = 10
    for _ in range(reps):
        tally.index_add_(0, idx, val)
    e.record()
    torch.cuda.synchronize(dev)
    return n * reps / (s.elapsed_time(e) * 1e-3)


PROFILE_SLAB = "electron_transport_slab64.md"
PROFILE_REQUESTS = "electron_requests_beamlets_ct128.md"


def ncu_figure(name, key):
    """A per-event figure (`key: value` line) of a committed ncu summary."""
    p = REPO / "profiles" / name
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":")[1].split()[0])
            except ValueError:
                return None
    return None


def ncu_traffic_per_event():
    """DRAM bytes per electron event from the committed ncu summary of the
    slab case."""
    return ncu_figure(PROFILE_SLAB, "dram_bytes_per_event")


def reference_rate(root, ph, spec_path, ncase, cores):
    """ompMC CLI (oracle/_ref) on `cores` host cores; histories/s of its batch loop."""
    from oracle import ref
    from ompmc_b200 import assets as A
    work = root / "bench"
    work.mkdir(parents=True, exist_ok=True)
    pf = work / "slab64.egsphant"
    if not pf.exists():
        A.write_egsphant(pf, ph)
    run = A.default_run(pf, ncase=ncase, nbatch=NBATCH, collimator=COLLIMATOR, output_folder=str(work) + "/")
    base = work / f"ref_{ncase}"
    A.write_inp(base, run)
    loop_s, _ = ref.run_cli(base, f"ref_{ncase}", cores=cores)
    return ncase / loop_s, loop_s


GANTRY = [0.0, 51.0, 103.0, 154.0, 206.0, 257.0, 309.0]


def bench_serving(device, nbeamlets, load=0.7, seed=7, plain_sample=12, params=None):
    """The beamlet serving workload: dose-influence requests on the 128x128x96
    x 0.3 cm CT-like phantom, 7 coplanar beams, 0.5x0.5 cm2 bixels at the
    isocentre (SAD 100 cm), histories per beamlet log-uniform in
    [2e4, 2e5], Poisson arrivals offered at `load` x measured capacity.
    Returns latency percentiles and throughput of the served event form and
    the plain FP64 form on a sample of the same beamlets (run one after the
    other, as the reference does).  `params`: event-form parameters
    (Engine.event_params keywords) set before the server is created."""
    from ompmc_b200 import assets as A
    from ompmc_b200.engine import PLAIN_FP64, Engine, Server, Tables, bixel_grid, load_spectrum
    root = A.require_assets()
    ph = A.ct_phantom(128, 128, 96, 0.3, seed=1234)
    spec = load_spectrum(root / "spectra" / "6mv.spectrum")
    eng = Engine(Tables.from_assets(A.CT_MEDIA, root), ph, device=device)
    if params:
        eng.event_params(**params)
    bl = bixel_grid(ph, GANTRY, bixel=0.5, field=(8.5, 8.5))        # 7 x 17 x 17 = 2023 bixels
    bl["spectrum"] = spec
    rng = np.random.default_rng(seed)
    nb_all = len(bl["corner"])
    pick = rng.choice(nb_all, size=min(nbeamlets, nb_all), replace=False)
    nh = np.exp(rng.uniform(np.log(2e4), np.log(2e5), size=len(pick))).astype(np.int64) // 10 * 10
    srv = Server(eng, seed=seed)
    bs = srv.beamlet_set(bl)
    # capacity probe: 16 requests back to back, after one untimed warm-up
    # burst (the first launches of a process load the kernels); the median
    # of three bursts
    caps = []
    for rep in range(4):
        t0 = time.perf_counter()
        ids = [srv.submit_beamlet(bs, int(pick[(i + 16 * rep) % len(pick)]), 50000, 10, 1e-4) for i in range(16)]
        while srv.step(8) > 0:
            pass
        if rep > 0:
            caps.append(16 * 50000 / (time.perf_counter() - t0))
        for r in ids:
            srv.release(r)
    cap_hps = float(np.median(caps))
    rate = load * cap_hps / float(nh.mean())                            # requests per second
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(pick)))
    sub = {}
    t_start = time.perf_counter()
    k = 0
    guard = 0
    while True:
        now = time.perf_counter() - t_start
        while k < len(pick) and arrivals[k] <= now:
            # the time between arrival and submission counts as latency
            sub[k] = (srv.submit_beamlet(bs, int(pick[k]), int(nh[k]), 10, 1e-4), 1e3 * (now - arrivals[k]))
            k += 1
        active = srv.step(4)
        if active == 0:
            if k == len(pick):
                break
            time.sleep(max(0.0, min(0.002, arrivals[k] - (time.perf_counter() - t_start))))
        guard += 1
        if guard > 10_000_000:
            raise RuntimeError("serving bench did not drain")
    makespan = time.perf_counter() - t_start
    lat = np.array([srv.poll(r) + lag for r, lag in sub.values()])
    nnz = [len(srv.result_sparse(r)[0]) for r, _ in sub.values()]
    srv.close()
    served = float(nh.sum()) / makespan
    # plain FP64 history-based form, beamlets one after the other
    sample = {k: bl[k] for k in ("src", "corner", "side1", "side2", "ibeam")}
    m = min(plain_sample, len(pick))
    sample.update(corner=bl["corner"][pick[:m]], side1=bl["side1"][pick[:m]], side2=bl["side2"][pick[:m]],
                  ibeam=bl["ibeam"][pick[:m]], spectrum=spec)
    _, _, _, _, pst = eng.run_beamlets(sample, 50000, 10, 1e-4, seed=3, mode=PLAIN_FP64)
    plain = pst["histories"] / pst["seconds"]
    eng.close()
    return {"workload": "ct128x128x96 x 0.3 cm, 7 coplanar beams, 0.5x0.5 cm2 bixels, log-uniform 2e4-2e5 "
                        "histories, Poisson arrivals", "requests": len(pick), "histories": int(nh.sum()),
            "offered_load_frac": load, "capacity_hist_per_s": cap_hps, "served_hist_per_s": served,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_nnz_per_column": float(np.mean(nnz)), "plain_fp64_hist_per_s": plain,
            "speedup_served_vs_plain": served / plain}


def bench_served_beams(eng, spec, nhist, nreq):
    """The bench's dose runs as `nreq` beam requests submitted together to
    the continuous-batching server on the same (tuned) engine: the requests
    share the particle queues, so one request's last particles overlap the
    next one's injection and only the last request pays the end-of-run
    tail.  Wall-clock histories/s from submission to the last request's
    dose and uncertainty in host memory, after one untimed request."""
    from ompmc_b200.engine import Server
    srv = Server(eng, seed=11)
    try:
        r = srv.submit_beam(max(nhist // 10, NBATCH), NBATCH, spectrum=spec, collimator=COLLIMATOR)
        while srv.step(16) > 0:
            pass
        srv.release(r)
        t0 = time.perf_counter()
        ids = [srv.submit_beam(nhist, NBATCH, spectrum=spec, collimator=COLLIMATOR) for _ in range(nreq)]
        while srv.step(16) > 0:
            pass
        wall = time.perf_counter() - t0
        lat = [srv.poll(i) for i in ids]
        dose, unc = srv.result_dense(ids[-1])
        unc1 = mean_unc_above_half(dose.ravel(), unc.ravel())
        for i in ids:
            srv.release(i)
    finally:
        srv.close()
    return {"value": nreq * nhist / wall, "unit": "histories/s", "requests": nreq, "histories_per_request": nhist,
            "wall_s": wall, "first_done_ms": min(lat), "last_done_ms": max(lat),
            "mean_rel_unc_gt50pct_dmax": unc1}


def trace_phases(rows):
    """Phases of a profiled run from its per-cycle trace (rows of injected,
    photons, electrons, source ms, photon ms, electron ms): the cycles up to
    the last injection, the cycles after it, and the drain (a last row with
    no source or photon time)."""
    rows = np.asarray(rows, dtype=np.float64).reshape(-1, 6)
    ms = rows[:, 3:].sum(axis=1)
    drained = len(rows) > 1 and rows[-1, 3] == 0 and rows[-1, 4] == 0
    nc = len(rows) - (1 if drained else 0)
    inj = np.nonzero(rows[:nc, 0] > 0)[0]
    li = int(inj[-1]) if len(inj) else -1
    return {"cycles": nc, "last_injection_cycle": li, "injection_ms": float(ms[:li + 1].sum()),
            "after_injection_ms": float(ms[li + 1:nc].sum()), "drain_ms": float(rows[-1, 5]) if drained else 0.0,
            "drain_particles": int(rows[-1, 1] + rows[-1, 2]) if drained else 0}


def reduce_max(vals, dist, device):
    """Element-wise maximum over ranks (the job's time is its slowest rank)."""
    if dist is None:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def rank_seed(rank):
    """Base seed of a rank's histories: every rank (replica) gets its own."""
    return 1000003 * (rank + 1)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if getattr(args, "workload", "slab64") == "beamlets":
        return run_reference_beamlets(args)
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs an ompMC checkout at build time)"}))
        return 0
    root, ph, spec = workload_inputs()
    cores = host_cores()
    sample = args.ref_sample
    for _ in range(args.warmup):
        reference_rate(root, ph, spec, sample // 4, cores)
    rates, secs = [], []
    for _ in range(args.steps):
        r, s = reference_rate(root, ph, spec, sample, cores)
        rates.append(r)
        secs.append(s)
    total = sample * args.steps
    value = total / sum(secs)
    out = {
        "metric": METRIC, "value": value, "unit": "histories/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * sum(secs) / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": SLAB_WORKLOAD, "sample_histories_per_step": sample, "parallelism": f"openmp{cores}"},
        "cpu_baseline": {"value": value, "unit": "histories/s", "cores": cores, "kind": "reference",
                         "sample": f"{sample} histories x {args.steps} runs of the ompMC CLI (slab64)"},
        "e2e": {"value": value, "unit": "histories/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# --------------------------------------------------------------------------
# The served beamlet load (the headline workload)
# --------------------------------------------------------------------------
def serve_load(srv, load, rate, seed, idx=None, cycles=8):
    """One pass of the beamlet load through the server: the requests
    `order[idx]` submitted at the arrival times of a Poisson process of
    `rate` requests/s, each finished request's sparse column (rows, dose,
    variance) copied into host memory as soon as the server reports it.
    The beamlet set is uploaded at the first submission of the pass.
    Returns histories, device ms of the pass (events on the server's
    stream), wall seconds, latency from arrival and from submission (ms),
    column uncertainty and histories per request, result bytes, and the
    server's kernel launches during the pass."""
    from ompmc_b200.workloads import LOAD_NBATCH, LOAD_REL, column_unc
    order, nh, gaps = load["order"], load["nhist"], load["gaps"]
    if idx is None:
        idx = np.arange(len(order))
    arrivals = np.cumsum(gaps[idx]) / rate
    arrivals -= arrivals[0]
    bl = dict(load["beamlets"], spectrum=load["spectrum"])
    bs = srv.beamlet_set(bl)
    st0 = srv.stats()
    n = len(idx)
    sub, out = {}, {}
    k = 0
    srv.timer_start()
    t0 = time.perf_counter()
    for guard in range(50_000_000):
        now = time.perf_counter() - t0
        while k < n and arrivals[k] <= now:
            b = int(order[idx[k]])
            rid = srv.submit_beamlet(bs, b, int(nh[idx[k]]), LOAD_NBATCH, LOAD_REL, seed=seed * 100003 + b + 1)
            sub[rid] = (k, 1e3 * (now - arrivals[k]))
            k += 1
        active = srv.step(cycles)
        for rid in srv.completed():
            rows, vals, var = srv.result_sparse(rid)
            out[rid] = (srv.poll(rid), column_unc(vals, var), len(rows))
            srv.release(rid)
        if active == 0:
            if k == n:
                break
            time.sleep(max(0.0, min(0.002, arrivals[k] - (time.perf_counter() - t0))))
    else:
        raise RuntimeError("serving pass did not finish")
    dev_ms = srv.timer_stop()
    wall = time.perf_counter() - t0
    st1 = srv.stats()
    lat_sub = np.array([out[r][0] for r in sub])
    lat = lat_sub + np.array([sub[r][1] for r in sub])
    unc = np.array([out[r][1] for r in sub])
    hist = np.array([nh[idx[sub[r][0]]] for r in sub], dtype=np.float64)
    nnz = np.array([out[r][2] for r in sub], dtype=np.float64)
    return dict(histories=float(hist.sum()), dev_ms=dev_ms, wall_s=wall, lat_ms=lat, lat_sub_ms=lat_sub, unc=unc,
                nhist=hist, d2h_bytes=float(nnz.sum() * (4 + 8 + 8)), nnz=nnz,
                launches=st1["launches"] - st0["launches"], cycles=st1["cycles"] - st0["cycles"])


def unc_summary(unc, nhist, rate):
    """Uncertainty of a set of beamlet columns: the mean relative
    uncertainty above 50 % of each column's maximum, the per-history
    relative variance (unc^2 * histories, which the histories needed for 1 %
    divide by 1e-4), and the seconds to 1 % for one average beamlet at
    `rate` histories/s."""
    ok = np.isfinite(unc)
    q = unc[ok] ** 2 * nhist[ok]
    return {"mean_rel_unc_gt50pct_dmax": float(np.mean(unc[ok])), "rel_var_x_histories": float(np.mean(q)),
            "histories_to_1pct_per_beamlet": float(np.mean(q) / 1e-4),
            "seconds_to_1pct_per_beamlet": float(np.mean(q) / 1e-4 / rate), "beamlets": int(ok.sum())}


def beamlet_engine(load, device, profile=False, queue_capacity=0):
    from ompmc_b200.engine import Engine, Tables, load_spectrum
    from ompmc_b200 import assets as A
    load["spectrum"] = load_spectrum(load["spectrum_file"])
    eng = Engine(Tables.from_assets(load["media"], A.require_assets()), load["phantom"], ecut=0.7, pcut=0.01,
                 device=device, profile=profile, queue_capacity=queue_capacity)
    return eng


def main_beamlets(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from ompmc_b200.engine import PLAIN_FP64, Server
    from ompmc_b200.workloads import LOAD_NBATCH, LOAD_REL, beamlet_load
    load = beamlet_load(args.load_seed)
    eng = beamlet_engine(load, local)
    srv = Server(eng, seed=rank_seed(rank))
    seed0 = rank_seed(rank)
    rate = args.arrival_rate
    for i in range(args.warmup):
        serve_load(srv, load, rate, seed0 - 1 - i)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    passes = []
    for i in range(args.steps):
        passes.append(serve_load(srv, load, rate, seed0 + i))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    dev_s = sum(p["dev_ms"] for p in passes) * 1e-3
    wall = sum(p["wall_s"] for p in passes)
    dev_s, wall = reduce_max([dev_s, wall], dist, "cuda")
    total = sum(p["histories"] for p in passes) * world
    value = total / dev_s
    e2e = total / wall
    lat = np.concatenate([p["lat_ms"] for p in passes])
    lat_sub = np.concatenate([p["lat_sub_ms"] for p in passes])
    unc = np.concatenate([p["unc"] for p in passes])
    nh = np.concatenate([p["nhist"] for p in passes])
    launches = sum(p["launches"] for p in passes)
    nreq = len(load["order"])
    extras = {}
    if rank == 0:
        extras["unc"] = unc_summary(unc, nh, value)
        extras["saturated"] = {"arrival_rate_req_per_s": rate, "p50_ms": float(np.percentile(lat, 50)),
                               "p99_ms": float(np.percentile(lat, 99)),
                               "p50_ms_from_submission": float(np.percentile(lat_sub, 50)),
                               "p99_ms_from_submission": float(np.percentile(lat_sub, 99)),
                               "mean_nnz_per_column": float(np.mean(np.concatenate([p["nnz"] for p in passes])))}
        # latency under load: the same requests arriving at a fraction of
        # the measured throughput (Poisson), one untimed pass
        load_rate = args.latency_load * value / float(np.mean(load["nhist"]))
        lp = serve_load(srv, load, load_rate, seed0 + 5000, cycles=4)
        extras["latency_at_load"] = {"offered_load_frac": args.latency_load, "arrival_rate_req_per_s": load_rate,
                                     "served_hist_per_s": lp["histories"] / lp["wall_s"],
                                     "p50_ms": float(np.percentile(lp["lat_ms"], 50)),
                                     "p99_ms": float(np.percentile(lp["lat_ms"], 99))}
        # one request at a time, the reference's mode, on the beamlets of the
        # CPU baseline's sample
        sl, srate = serve_sequential(srv, load, args.ref_beamlets, seed0 + 7000)
        extras["sequential"] = {"requests": args.ref_beamlets, "p50_ms": float(np.percentile(sl, 50)),
                                "p99_ms": float(np.percentile(sl, 99)), "hist_per_s": srate,
                                "mode": "each request submitted when the previous column is in host memory"}
    srv.close()
    if rank == 0 and not args.no_extras and world == 1:
        extras.update(beamlet_extras(args, load, eng, value, local))
    eng.close()
    if rank == 0:
        d2h = float(np.mean([p["d2h_bytes"] for p in passes]))
        out = {
            "metric": METRIC, "value": value, "unit": "histories/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "p50_ms": extras.get("latency_at_load", {}).get("p50_ms"),
            "p99_ms": extras.get("latency_at_load", {}).get("p99_ms"),
            "config": {"workload": WORKLOAD, "requests_per_step": nreq,
                       "histories_per_step": float(np.sum(load["nhist"])),
                       "arrival_rate_req_per_s": rate, "nbatch": LOAD_NBATCH, "rel_threshold": LOAD_REL,
                       "mode": "event FP32 transport / FP64 tallies, served (continuous batching)",
                       "parallelism": f"replicas{world}", "load_seed": args.load_seed,
                       "l2": "particle queues (0.87 GB) and per-request batch tallies (126 MB each, up to 254 "
                             "requests resident) exceed L2; physics tables are L2-resident"},
            "e2e": {"value": e2e, "unit": "histories/s",
                    "h2d_bytes_per_step": int(4 * (3 * 7 + 9 * nreq + 2 * 1000) + 4 * nreq + 64 * nreq),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        out.update(extras)
        print(json.dumps(out))
    if dist:
        dist.destroy_process_group()
    return 0


def beamlet_extras(args, load, eng, value, device):
    """Roofline of the dominant kernel, the plain FP64 comparator and the CPU
    reference on samples of the same load (rank 0, one GPU, untimed)."""
    from ompmc_b200.engine import PLAIN_FP64, Server
    extras = {}
    peak, peak_kind = peaks()
    # a profiled pass over part of the load: per-kernel device time and
    # transport counters with the kernels launched one by one
    prof, hist, nsub = profiled_pass(load, device, args.profile_requests, args.arrival_rate)
    ek, pk = prof["electron"], prof["photon"]
    nl = max(1, ek["launches"])
    # table and voxel bytes the electron kernels request per event, counted
    # by ncu's SASS counters on this load (queue state excluded); the
    # code-read estimate of 10 table pair lookups per condensed-history step
    # + 3 per event is kept beside it
    req = ncu_figure(PROFILE_REQUESTS, "requested_bytes_per_event")
    est_bytes = 8 * ek["cross"] + 16 * ek["dep"] + 8 * (10 * ek["steps"] + 3 * ek["particles"])
    alg_bytes = (req - 104) * ek["particles"] if req else est_bytes
    achieved = alg_bytes / ek["seconds"] / 1e9
    tpe = ncu_figure(PROFILE_REQUESTS, "dram_bytes_per_event") or ncu_traffic_per_event()
    per_launch_events = ek["particles"] / nl
    total_s = sum(x["seconds"] for x in prof.values())
    extras["roofline"] = {
        "bound": "hbm", "kernel": "k_electron_step + k_electron_interact (+ k_drain)", "achieved": achieved,
        "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
        "traffic": (tpe * per_launch_events) if tpe else None,
        "algorithmic_bytes_per_launch": alg_bytes / nl,
        "algorithmic_bytes": "requested by the kernels' global loads, stores and reductions (ncu SASS counters, "
                             "per event) less the 104 B of queue state" if req else
                             "8 B per voxel crossing + 16 B per deposit + 8 B per estimated table pair lookup",
        "estimated_bytes_per_launch": est_bytes / nl,
        "state_bytes_per_launch": 104 * per_launch_events,
        "avg_launch_ms": 1000 * ek["seconds"] / nl,
        "kernel_seconds": {k: v["seconds"] for k, v in prof.items()},
        "kernel_share": {k: v["seconds"] / max(1e-12, total_s) for k, v in prof.items()},
        "sample": f"profiled pass over {nsub} requests of the load",
    }
    extras["per_history"] = {k: (ek[k] + pk[k]) / hist for k in ("particles", "steps", "cross", "dep", "atom")}
    # plain FP64 history-based form on a sample of the same beamlets, one
    # after the other (omc_run_beamlets)
    m = args.plain_sample
    pick = load["order"][:m]
    bl = load["beamlets"]
    sample = dict(src=bl["src"], corner=bl["corner"][pick], side1=bl["side1"][pick], side2=bl["side2"][pick],
                  ibeam=bl["ibeam"][pick], spectrum=load["spectrum"])
    nplain = int(np.mean(load["nhist"]))
    eng.run_beamlets(sample, nplain // 10, 10, 1e-4, seed=2, mode=PLAIN_FP64)
    _, _, _, _, pst = eng.run_beamlets(sample, nplain, 10, 1e-4, seed=3, mode=PLAIN_FP64)
    plain = pst["histories"] / pst["seconds"]
    extras["plain_fp64"] = {"value": plain, "unit": "histories/s", "beamlets": m, "histories_per_beamlet": nplain,
                            "speedup_served_vs_plain": value / plain}
    # the reference (unmodified matRad entry, OpenMP) on this host's cores
    from oracle import refbench
    if refbench.available():
        cores = host_cores()
        res = refbench.run_pinned(load["order"][:args.ref_beamlets], load["nhist"][:args.ref_beamlets], cores,
                                  seed=args.load_seed)
        r = ref_summary(res)
        extras["cpu_baseline"] = {"value": r["value"], "unit": "histories/s", "cores": cores, "kind": "reference",
                                  "sample": f"{len(res)} beamlets of the load, one unmodified matRad-entry call each "
                                            f"(OpenMP), {r['loop_s']:.1f} s of beamlet loops",
                                  "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "unc": r["unc"]}
        one = refbench.run_pinned(load["order"][:args.ref_beamlets_1core], load["nhist"][:args.ref_beamlets_1core],
                                  1, seed=args.load_seed)
        r1 = ref_summary(one)
        extras["cpu_baseline_1core"] = {"value": r1["value"], "unit": "histories/s", "cores": 1, "kind": "reference",
                                        "sample": f"{len(one)} beamlets, {r1['loop_s']:.1f} s"}
    else:
        extras["cpu_baseline"] = None
    return extras


def profiled_pass(load, device, nreq, rate, max_requests=0, queue_capacity=0):
    """The first `nreq` requests of the load through a server whose engine
    launches every kernel on its own with events around it and counts
    transport events (particles), condensed-history steps, voxel crossings,
    deposits and tally atomics per kernel.  Returns those counters, the
    histories of the pass and the request count."""
    from ompmc_b200.engine import Server
    pe = beamlet_engine(load, device, profile=True, queue_capacity=queue_capacity)
    ps = Server(pe, seed=99, max_requests=max_requests)
    sub = np.arange(min(nreq, len(load["order"])))
    serve_load(ps, load, rate, 424242, idx=sub)
    prof = pe.profile_last()
    ps.close()
    pe.close()
    return prof, float(np.sum(load["nhist"][sub])), len(sub)


def serve_sequential(srv, load, n, seed, cycles=4):
    """The first `n` requests of the load served one at a time, the way the
    reference's matRad entry runs its beamlets: each request is submitted
    once the previous one's sparse column is in host memory.  Returns the
    latency of each request (ms, submission to column in host memory) and
    the histories/s of the sequence."""
    from ompmc_b200.workloads import LOAD_NBATCH, LOAD_REL
    bs = srv.beamlet_set(dict(load["beamlets"], spectrum=load["spectrum"]))
    lat = []
    t_all = time.perf_counter()
    for k in range(n):
        b = int(load["order"][k])
        t0 = time.perf_counter()
        srv.submit_beamlet(bs, b, int(load["nhist"][k]), LOAD_NBATCH, LOAD_REL, seed=seed * 100003 + b + 1)
        done = False
        for guard in range(10_000_000):
            srv.step(cycles)
            for rid in srv.completed():
                srv.result_sparse(rid)
                srv.release(rid)
                done = True
            if done:
                break
        else:
            raise RuntimeError("sequential request did not finish")
        lat.append(1e3 * (time.perf_counter() - t0))
    wall = time.perf_counter() - t_all
    return np.array(lat), float(np.sum(load["nhist"][:n])) / wall


def ref_summary(res):
    """Histories/s, per-beamlet time percentiles and uncertainty of the
    reference's beamlet runs (refbench records)."""
    nh = np.array([r["nhist"] for r in res], dtype=np.float64)
    ls = np.array([r["loop_s"] for r in res])
    unc = np.array([r["unc"] for r in res])
    value = float(nh.sum() / ls.sum())
    return {"value": value, "loop_s": float(ls.sum()), "p50_ms": float(np.percentile(1e3 * ls, 50)),
            "p99_ms": float(np.percentile(1e3 * ls, 99)), "unc": unc_summary(unc, nh, value)}


def run_reference_beamlets(args):
    """Reference arm on the beamlet load: the unmodified matRad entry on all
    host cores, a different sample of the load's beamlets each step (the
    same beamlets, in the same order, that the GPU arm serves), one call per
    beamlet as the per-request history counts need."""
    from oracle import refbench
    if not refbench.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs an ompMC checkout "
                                                               "at build time)"}))
        return 0
    from ompmc_b200.workloads import LOAD_NBATCH, LOAD_REL, beamlet_load
    load = beamlet_load(args.load_seed)
    order, nh = load["order"], load["nhist"]
    cores = host_cores()
    S = args.ref_beamlets_per_step
    n = len(order)
    for w in range(args.warmup):
        pos = np.array([n - 1 - w])
        refbench.run_pinned(order[pos], nh[pos], cores, seed=args.load_seed)
    res, per_step = [], []
    for k in range(args.steps):
        pos = (k * S + np.arange(S)) % n            # requests k*S .. k*S+S-1 of the load
        r = refbench.run_pinned(order[pos], nh[pos], cores, seed=args.load_seed)
        res += r
        per_step.append(sum(x["loop_s"] for x in r))
    s = ref_summary(res)
    out = {
        "metric": METRIC, "value": s["value"], "unit": "histories/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(per_step)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "p50_ms": s["p50_ms"], "p99_ms": s["p99_ms"],
        "config": {"workload": WORKLOAD, "beamlets_per_step": S, "nbatch": LOAD_NBATCH, "rel_threshold": LOAD_REL,
                   "parallelism": f"openmp{cores}", "load_seed": args.load_seed,
                   "timing": "the beamlet loop of each call (waitbar calls before and after it); table "
                             "initialisation per call excluded"},
        "cpu_baseline": {"value": s["value"], "unit": "histories/s", "cores": cores, "kind": "reference",
                         "sample": f"{S} beamlets of the load per step x {args.steps} steps, unmodified matRad "
                                   f"entry (OpenMP)"},
        "e2e": {"value": s["value"], "unit": "histories/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "unc": s["unc"],
    }
    print(json.dumps(out))
    return 0


def main_slab64(args):
    serving_params = json.loads(args.serving_params) if args.serving_params else None
    if args.serving_only:
        print(json.dumps({"serving": bench_serving(int(os.environ.get("LOCAL_RANK", "0")), args.serving_requests,
                                                   params=serving_params), "params": serving_params}))
        return 0

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from ompmc_b200.engine import EVENT_FP32, PLAIN_FP64, Engine, Tables, load_spectrum
    root, ph, spec_path = workload_inputs()
    spec = load_spectrum(spec_path)
    tables = Tables.from_assets(MEDIA, root)
    eng = Engine(tables, ph, ecut=0.7, pcut=0.01, device=local)
    mode = EVENT_FP32 if args.mode == "event" else PLAIN_FP64
    nstep = args.hist_per_step
    seed0 = rank_seed(rank)

    # results land in pinned host buffers (the e2e copy is a DMA from the device)
    nv = int(np.prod(eng.shape))
    pinned = tuple(torch.empty(nv, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2))

    def step(i, e=eng, m=mode, n=nstep):
        return e.run_beam(n, NBATCH, seed=seed0 + i, mode=m, spectrum=spec, collimator=COLLIMATOR,
                          out=pinned if e is eng else None)

    if args.cycle_trace:
        # same seed as the first warm-up step: the queue sizes per cycle are
        # those of the launches a profiler sees first
        te = Engine(tables, ph, ecut=0.7, pcut=0.01, device=local, profile=True)
        if serving_params:
            te.event_params(**serving_params)
        # untimed small run first: the first launches of a process load the kernels
        te.run_beam(max(nstep // 10, NBATCH), NBATCH, seed=seed0 - 2, mode=EVENT_FP32, spectrum=spec,
                    collimator=COLLIMATOR)
        te.run_beam(nstep, NBATCH, seed=seed0 - 1, mode=EVENT_FP32, spectrum=spec, collimator=COLLIMATOR)
        rows = te.profile_trace()
        drain = te.profile_drain()
        te.close()
        cols = ["injected", "photons", "electrons", "source_ms", "photon_ms", "electron_ms"]
        phases = dict(trace_phases(rows), drain=drain)
        print(json.dumps({"seed": seed0 - 1, "histories": nstep, "params": serving_params, "phases": phases,
                          "columns": cols, "cycles": rows.tolist()}))
        eng.close()
        return 0
    tuned = None
    if not args.no_tune:
        # launch parameters picked by the autotuner on 3*10^6-history runs of
        # the same beam (untimed; results do not depend on them); shorter
        # runs over-weight the end of a run, where other settings win
        from ompmc_b200.autotune import tune_beam
        cfg, rate, trials = tune_beam(eng, nhist=min(nstep, 3_000_000), repeats=3, spectrum=spec,
                                      collimator=COLLIMATOR)
        tuned = dict(cfg, trials=len(trials), tune_hist_per_s=rate)
    for i in range(args.warmup):
        step(-1 - i)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    t0 = time.perf_counter()
    dev_s = 0.0
    launches = 0
    uncs = []
    for i in range(args.steps):
        dose, unc, st = step(i)
        dev_s += st["seconds"]
        launches += st["launches"]
        uncs.append(mean_unc_above_half(dose, unc))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    dev_s, wall = reduce_max([dev_s, wall], dist, "cuda")
    total = nstep * args.steps * world
    value = total / dev_s
    e2e = total / wall
    nvox = int(np.prod(eng.shape))

    extras = {}
    if rank == 0:
        # roofline of the dominant kernel from a profiled (untimed) step
        peak, peak_kind = peaks()
        prof_eng = Engine(tables, ph, ecut=0.7, pcut=0.01, device=local, profile=True)
        if tuned:
            prof_eng.event_params(**{k: tuned[k] for k in ("electron_tsteps", "tail_boost", "inflight", "block",
                                                           "electron_split", "electron_chsteps",
                                                           "drain_particles")})
        prof_eng.run_beam(nstep, NBATCH, seed=777, mode=EVENT_FP32, spectrum=spec, collimator=COLLIMATOR)
        prof = prof_eng.profile_last()
        prof_eng.close()
        ek = prof["electron"]
        pk = prof["photon"]
        lookups = 10 * ek["steps"] + 3 * ek["particles"]
        alg_bytes = 8 * ek["cross"] + 16 * ek["dep"] + 8 * lookups
        achieved = alg_bytes / ek["seconds"] / 1e9
        tpe = ncu_traffic_per_event()
        per_launch_events = ek["particles"] / max(1, ek["launches"])
        extras["roofline"] = {
            "bound": "hbm", "kernel": "k_electron_step + k_electron_interact + k_drain", "achieved": achieved,
            "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": (tpe * per_launch_events) if tpe else None,
            "algorithmic_bytes_per_launch": alg_bytes / max(1, ek["launches"]),
            # particle-state queue traffic, reported apart from the algorithmic
            # figure: 52 B loaded and 52 B stored per electron event
            "state_bytes_per_launch": 104 * per_launch_events,
            "achieved_with_state": (alg_bytes + 104 * ek["particles"]) / ek["seconds"] / 1e9,
            "avg_launch_ms": 1000 * ek["seconds"] / max(1, ek["launches"]),
            "kernel_seconds": {k: v["seconds"] for k, v in prof.items()},
            "kernel_share": {k: v["seconds"] / max(1e-12, sum(x["seconds"] for x in prof.values()))
                             for k, v in prof.items()},
        }
        hist = nstep
        per_hist = {k: ek[k] / hist + pk[k] / hist for k in ("particles", "steps", "cross", "dep", "atom")}
        try:
            apk = atomic_peak(local, nvox)
            atom_rate = (ek["atom"] + pk["atom"]) / (ek["seconds"] + pk["seconds"])
            extras["atomics"] = {"tally_atomics_per_s_in_kernels": atom_rate, "measured_fp64_scatter_peak": apk,
                                 "frac": atom_rate / apk}
        except Exception as ex:  # the torch microbenchmark is optional
            extras["atomics"] = {"error": str(ex)[:200]}
        extras["per_history"] = per_hist
        unc1 = float(np.mean(uncs))
        extras["dose_unc"] = {"mean_rel_unc_gt50pct_dmax": unc1, "histories_per_step": nstep,
                              "histories_to_1pct": nstep * (unc1 / 0.01) ** 2,
                              "seconds_to_1pct": nstep * (unc1 / 0.01) ** 2 / value}
        if not args.no_extras and world == 1:
            # plain FP64 history-based form on the same workload (comparator)
            pn = max(nstep // 5, 100000)
            step(999, m=PLAIN_FP64, n=pn)
            _, _, pst = step(1000, m=PLAIN_FP64, n=pn)
            plain = pn / pst["seconds"]
            extras["plain_fp64"] = {"value": plain, "unit": "histories/s", "speedup_event_vs_plain": value / plain}
            # photon splitting (nsplit = 20, the reference's sample input):
            # fewer histories/s, lower variance per history; compared by the
            # time to 1 % mean uncertainty in voxels above 50 % of the maximum
            sn = max(nstep // 4, 100000)
            se = Engine(tables, ph, ecut=0.7, pcut=0.01, device=local, nsplit=20)
            step(998, e=se, n=sn)
            sd, su, sst = step(997, e=se, n=sn)
            se.close()
            su1 = mean_unc_above_half(sd, su)
            srate = sn / sst["seconds"]
            extras["nsplit20"] = {"value": srate, "unit": "histories/s", "histories": sn,
                                  "mean_rel_unc_gt50pct_dmax": su1,
                                  "seconds_to_1pct": sn * (su1 / 0.01) ** 2 / srate}
            # CPU reference on this host's cores (bounded sample)
            from oracle import ref
            if ref.available():
                cores = host_cores()
                r, s = reference_rate(root, ph, spec_path, args.ref_sample, cores)
                extras["cpu_baseline"] = {"value": r, "unit": "histories/s", "cores": cores, "kind": "reference",
                                          "sample": f"{args.ref_sample} histories of the slab64 workload, ompMC CLI, "
                                                    f"{s:.1f} s batch loop"}
            else:
                extras["cpu_baseline"] = None
        if args.serving_requests > 0 and world == 1:
            extras["serving"] = bench_serving(local, args.serving_requests, params=serving_params)
        if not args.no_extras and world == 1 and mode == EVENT_FP32:
            extras["served_beams"] = bench_served_beams(eng, spec, nstep, args.steps)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "histories/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if mode == EVENT_FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": SLAB_WORKLOAD, "mode": args.mode, "histories_per_step_per_gpu": nstep,
                       "tally": "f64", "parallelism": f"replicas{world}", "tuned": tuned,
                       "l2": "particle queues (0.8 GB) and batch tallies exceed L2; physics tables are L2-resident"},
            "e2e": {"value": e2e, "unit": "histories/s", "h2d_bytes_per_step": 2 * 1000 * 8 + 64,
                    "d2h_bytes_per_step": 2 * nvox * 8},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        out.update(extras)
        print(json.dumps(out))
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="beamlets", choices=["beamlets", "slab64"])
    ap.add_argument("--no-extras", action="store_true", help="skip the comparators (CPU reference, plain form)")
    # beamlet load
    ap.add_argument("--load-seed", type=int, default=7, help="seed of the request order, histories and arrivals")
    ap.add_argument("--arrival-rate", type=float, default=4000.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--latency-load", type=float, default=0.7,
                    help="offered load of the latency pass, as a fraction of the measured throughput")
    ap.add_argument("--profile-requests", type=int, default=400, help="requests of the profiled pass")
    ap.add_argument("--plain-sample", type=int, default=12, help="beamlets of the plain FP64 comparator")
    ap.add_argument("--ref-beamlets", type=int, default=24, help="beamlets of the CPU baseline (all cores)")
    ap.add_argument("--ref-beamlets-1core", type=int, default=2, help="beamlets of the 1-core CPU baseline")
    ap.add_argument("--ref-beamlets-per-step", type=int, default=16, help="reference arm: beamlets per step")
    # slab64 dose run
    ap.add_argument("--mode", default="event", choices=["event", "plain"])
    ap.add_argument("--hist-per-step", type=int, default=HIST_PER_STEP)
    ap.add_argument("--ref-sample", type=int, default=10_000_000)
    ap.add_argument("--serving-requests", type=int, default=300,
                    help="slab64: beamlet requests in the serving extra (0 skips it)")
    ap.add_argument("--no-tune", action="store_true", help="slab64: skip the autotuner (default launch parameters)")
    ap.add_argument("--cycle-trace", action="store_true",
                    help="slab64: print the per-cycle trace (queue sizes, kernel ms) of the first warm-up step and "
                         "exit")
    ap.add_argument("--serving-only", action="store_true",
                    help="run only the 300-request serving sample and print its JSON object")
    ap.add_argument("--serving-params", default=None,
                    help="event-form parameters of the serving engine (and of the --cycle-trace run), as JSON "
                         "(Engine.event_params keywords)")
    ap.add_argument("--profiled-pass", action="store_true",
                    help="beamlets: run only the profiled pass over --profile-requests requests (the case of the "
                         "ncu capture of the electron kernel's requested bytes) and print its counters")
    ap.add_argument("--profile-max-requests", type=int, default=0,
                    help="profiled pass: requests resident at once (0: as the memory budget allows)")
    ap.add_argument("--profile-queue-capacity", type=int, default=0,
                    help="profiled pass: particle queue capacity (0: the engine's default)")
    args = ap.parse_args()
    if args.profiled_pass:
        from ompmc_b200.workloads import beamlet_load
        prof, hist, nsub = profiled_pass(beamlet_load(args.load_seed), int(os.environ.get("LOCAL_RANK", "0")),
                                         args.profile_requests, args.arrival_rate, args.profile_max_requests,
                                         args.profile_queue_capacity)
        print(json.dumps({"requests": nsub, "histories": hist, "counters": prof}))
        return 0
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "slab64" or args.serving_only or args.cycle_trace:
        return main_slab64(args)
    return main_beamlets(args)


if __name__ == "__main__":
    sys.exit(main())
