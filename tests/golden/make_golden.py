"""Generates the golden fixtures in this directory from the unmodified
reference (built by oracle/Makefile) — run here, where an ompMC checkout
exists; the fixtures are committed so GPU hosts need neither.

    python tests/golden/make_golden.py [--only NAME]

Fixtures (all seeded; reference RNG seeds 97 33, one thread):
  rays_<case>.npz     random rays and the reference howfar walk of each
                      (ustep, irnew, idisc per call) and hownear at start
  replay_<case>.npz   primaries, the uniform stream each history consumed
                      (stored exactly as integers rn * 2^24, RANMAR's
                      resolution) and its deposit sequence (region, energy)
  replaysplit_<case>.npz  the same with photon splitting, nsplit = 20
  replayspin_<case>.npz   the same with the synthetic, non-constant spin file
                      (assets.write_spin_synthetic; data folder data_spin)
  kat_<case>.npz      known answers of every interaction sampler and of
                      msdist: seeded particles in random voxels, scripted
                      streams, the reference's output particles and
                      random-number counts (katspin_: with the synthetic spin
                      file, which the MS sampler inside msdist reads)
  dose*_<case>.npz    reference CLI dose and relative uncertainty of the
                      voxels above 5 % of the maximum (8 threads, 50 batches;
                      sources in DOSE: 6 MV and 18 MV photon spectra, 6 MeV
                      electrons, 3 MeV positrons; dosesplit: 6 MV with
                      photon splitting, nsplit = 20)
  gamma_<case>.npz    high-statistics reference CLI dose of the voxels above
                      2 % of the maximum for the gamma 2 %/2 mm test (8 threads;
                      water30 1e8, slab64 4e8 histories in 100 batches)
  (the table comparison runs against the live oracle; no fixture)
Cases: water30 (30^3 x 1 cm water), slab64 (64^3 x 0.25 cm water/lung/bone),
ctsmall (32x32x24 x 1.2 cm CT-like, 4 media).
"""
from __future__ import annotations

import argparse
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))

from ompmc_b200 import assets as A  # noqa: E402

WORK = REPO / "assets" / "golden_work"
SPLIT = 20      # photon splitting factor of the *split* fixtures (the sample input's value)

CASES = {
    "water30": dict(phantom=lambda: A.water_cube(30, 1.0), collimator=(-5, 5, -5, 5)),
    "slab64": dict(phantom=lambda: A.slab_phantom(64, 0.25), collimator=(-2.5, 2.5, -2.5, 2.5)),
    "ctsmall": dict(phantom=lambda: A.ct_phantom(32, 32, 24, 1.2, seed=7), collimator=(-5, 5, -5, 5)),
}

TABLES = ["ge0", "ge1", "gmfp0", "gmfp1", "gbr10", "gbr11", "gbr20", "gbr21", "cohe0", "cohe1", "xgrid", "fcum",
          "b_array", "c_array", "pmax0", "pmax1", "i_array", "dl1", "dl2", "dl3", "dl4", "dl5", "dl6", "bpar0",
          "bpar1", "delcm", "zbrang", "esig0", "esig1", "psig0", "psig1", "ededx0", "ededx1", "pdedx0", "pdedx1",
          "ebr10", "ebr11", "pbr10", "pbr11", "pbr20", "pbr21", "tmxs0", "tmxs1", "blcce0", "blcce1", "etae_ms0",
          "etae_ms1", "etap_ms0", "etap_ms1", "q1ce_ms0", "q1ce_ms1", "q1cp_ms0", "q1cp_ms1", "q2ce_ms0",
          "q2ce_ms1", "q2cp_ms0", "q2cp_ms1", "range_ep", "e_array", "eke0", "eke1", "sig_ismonotone", "esig_e",
          "psig_e", "xcc", "blcc", "expeke1", "spin_rej", "ums", "fms", "wms", "ims", "meke"]


def case_inp(name, ncase=100000, nbatch=10, nsplit=1, spin=False):
    """Phantom + spectrum + `.inp` of a case under assets/golden_work.
    spin: the data folder with the synthetic (non-constant) spin file."""
    A.require_assets()
    c = CASES[name]
    ph = c["phantom"]()
    pf = WORK / f"{name}.egsphant"
    if not pf.exists():
        A.write_egsphant(pf, ph)
    run = A.default_run(pf, ncase=ncase, nbatch=nbatch, collimator=c["collimator"])
    run.nsplit = nsplit
    if spin:
        run.data_folder = str(A.stage_spin_variant()) + "/"
    base = WORK / (f"{name}_{ncase}" if nsplit == 1 else f"{name}_{ncase}_split{nsplit}")
    if spin:
        base = base.with_name(base.name + "_spin")
    A.write_inp(base, run)
    return base, ph


def random_rays(ph, n, rng):
    """Rays starting inside random voxels, isotropic directions."""
    nx, ny, nz = ph.shape
    i = rng.integers(0, nx, n)
    j = rng.integers(0, ny, n)
    k = rng.integers(0, nz, n)
    fx, fy, fz = rng.random((3, n))
    x = ph.xb[i] + fx * (ph.xb[i + 1] - ph.xb[i])
    y = ph.yb[j] + fy * (ph.yb[j + 1] - ph.yb[j])
    z = ph.zb[k] + fz * (ph.zb[k + 1] - ph.zb[k])
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    # a few axis-aligned rays exercise the zero-cosine branches
    d[: n // 10] = np.eye(3)[rng.integers(0, 3, n // 10)] * rng.choice([-1, 1], (n // 10, 1))
    ir = 1 + i + j * nx + k * nx * ny
    return np.column_stack([x, y, z, d, ir]).astype(np.float64)


def _in_subprocess(name, what, out):
    """The reference keeps global state: one configuration per process."""
    code = (f"import sys; sys.path.insert(0, {str(REPO)!r}); sys.argv=['x']; "
            f"from tests.golden import make_golden as M; M._{what}({name!r}, {str(out)!r})")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError(p.stdout[-3000:] + p.stderr[-3000:])


def _rays(name, out):
    from oracle.ref import Reference
    base, ph = case_inp(name)
    r = Reference.open(base)
    rays = random_rays(ph, 300, np.random.default_rng(11))
    cap = 4 * sum(ph.shape)
    us = np.zeros((len(rays), cap))
    irn = np.zeros((len(rays), cap), dtype=np.int32)
    idc = np.zeros((len(rays), cap), dtype=np.int32)
    nc = np.zeros(len(rays), dtype=np.int32)
    hn = np.zeros(len(rays))
    for q, ray in enumerate(rays):
        a, b, c = r.walk(*ray[:6], int(ray[6]), cap=cap)
        n = len(a)
        us[q, :n], irn[q, :n], idc[q, :n], nc[q] = a, b, c, n
        hn[q] = r.hownear(*ray[:3], int(ray[6]))
    np.savez_compressed(out, rays=rays, ustep=us, irnew=irn, idisc=idc, ncalls=nc, hownear=hn, cap=cap)


def _replay(name, out, spin=False):
    from oracle.ref import Reference
    base, _ = case_inp(name, spin=spin)
    r = Reference.open(base)
    nh = {"water30": 200, "slab64": 150, "ctsmall": 150}[name]
    res = r.run(nh)
    rn_int = np.round(res["rn"] * 16777216.0).astype(np.uint32)
    assert np.array_equal(rn_int.astype(np.float64) / 16777216.0, res["rn"])
    np.savez_compressed(out, prim=res["prim"], rn_int=rn_int, rn_off=res["rn_off"], dep_ir=res["dep_ir"],
                        dep_e=res["dep_e"], d_off=res["d_off"])


def _replaysplit(name, out):
    """As _replay, with photon splitting (nsplit = SPLIT) and the Russian
    roulette of photons from electron interactions."""
    from oracle.ref import Reference
    base, _ = case_inp(name, nsplit=SPLIT)
    r = Reference.open(base)
    nh = 40
    res = r.run(nh, rn_cap=nh * 60000, dep_cap=nh * 6000)
    rn_int = np.round(res["rn"] * 16777216.0).astype(np.uint32)
    assert np.array_equal(rn_int.astype(np.float64) / 16777216.0, res["rn"])
    np.savez_compressed(out, prim=res["prim"], rn_int=rn_int, rn_off=res["rn_off"], dep_ir=res["dep_ir"],
                        dep_e=res["dep_e"], d_off=res["d_off"], nsplit=SPLIT)


def _replayspin(name, out):
    """As _replay, with the synthetic spin file (spin rejection and the MS
    moment corrections active)."""
    _replay(name, out, spin=True)


def _tables(name, out, spin=False):
    from oracle.ref import Reference
    base, _ = case_inp(name, spin=spin)
    r = Reference.open(base)
    d = {n: r.table(n) for n in TABLES}
    for k, v in r.spin_scalars().items():
        d["s_" + k] = np.array(v)
    np.savez_compressed(out, **d)


def _tablesspin(name, out):
    _tables(name, out, spin=True)


KAT_CASES = 120        # cases per sampler
KAT_STREAM = 4096      # uniforms offered per case (multiples of 2^-24)
RM = 0.5109989461


def kat_inputs(ph, which, n, rng):
    """Particles (x,y,z,u,v,w,e,wt,ir,iq,dnear; e total energy) for the
    sampler `which` (oracle.ref.Reference.SAMPLERS order, 9 = msdist) in
    random voxels of the phantom, and (de, tustep) for msdist."""
    nx, ny, nz = ph.shape
    i, j, k = rng.integers(0, nx, n), rng.integers(0, ny, n), rng.integers(0, nz, n)
    fx, fy, fz = rng.random((3, n))
    x = ph.xb[i] + fx * (ph.xb[i + 1] - ph.xb[i])
    y = ph.yb[j] + fy * (ph.yb[j + 1] - ph.yb[j])
    z = ph.zb[k] + fz * (ph.zb[k + 1] - ph.zb[k])
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    ir = 1 + i + j * nx + k * nx * ny
    logu = lambda lo, hi: np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    iq = np.zeros(n)
    if which == 0:
        e = logu(0.02, 18.0)                    # compton
    elif which == 1:
        e = logu(0.01, 1.0)                     # photo
    elif which == 2:
        e = logu(1.03, 18.0)                    # pair
    elif which == 3:
        e = logu(0.01, 2.0)                     # rayleigh
    elif which in (4, 6, 9):
        iq = -np.ones(n) if which == 4 else rng.choice([-1.0, 1.0], n)
        e = logu(0.05, 18.0) + RM               # moller, brems, msdist
    elif which in (5, 7):
        iq = np.ones(n)
        e = logu(0.05 if which == 5 else 0.01, 18.0) + RM   # bhabha, annih in flight
    else:
        iq = np.ones(n)
        e = np.full(n, RM)                      # rannih: at rest
    q = np.column_stack([x, y, z, d, e, np.ones(n), ir, iq, np.zeros(n)]).astype(np.float64)
    extra = None
    if which == 9:
        eke = e - RM
        rhof = ph.rho.ravel()[ir - 1]
        tustep = 10.0 ** rng.uniform(-3.5, -1.0, n) * eke / np.maximum(rhof, 1e-3)
        de = np.minimum(tustep * np.maximum(rhof, 1e-3) * 2.0 * rng.uniform(0.5, 1.5, n), 0.5 * eke)
        extra = np.column_stack([de, tustep])
    return q, extra


def _kat(name, out, spin=False):
    """Every interaction sampler and msdist on seeded particles and scripted
    streams: the reference's outputs and random-number counts."""
    from oracle.ref import Reference
    base, ph = case_inp(name, spin=spin)
    r = Reference.open(base)
    rng = np.random.default_rng(4711 + (1 if spin else 0))
    names = {v: k for k, v in Reference.SAMPLERS.items()}
    res = {}
    for which in range(10):
        q, extra = kat_inputs(ph, which, KAT_CASES, rng)
        streams, outs, nouts, used = [], [], [], []
        for c in range(KAT_CASES):
            rn_int = rng.integers(0, 1 << 24, KAT_STREAM, dtype=np.uint32)
            rn = rn_int.astype(np.float64) / 16777216.0
            o = np.zeros((4, 11))
            if which == 9:
                ustep, u, fin = r.msdist(q[c], extra[c, 0], extra[c, 1], rn)
                o[0, 0] = ustep
                o[0, 1:7] = fin
                nout = 1
            else:
                u, parts = r.sampler(names[which], q[c], rn)
                nout = len(parts)
                o[:nout] = parts
            if u < 0:
                raise RuntimeError(f"stream of {KAT_STREAM} numbers too short for sampler {which}")
            streams.append(rn_int[:u])
            outs.append(o)
            nouts.append(nout)
            used.append(u)
        off = np.concatenate([[0], np.cumsum([len(x) for x in streams])]).astype(np.int64)
        key = "msdist" if which == 9 else names[which]
        res[f"{key}_q"] = q
        if extra is not None:
            res[f"{key}_extra"] = extra
        res[f"{key}_rn_int"] = np.concatenate(streams).astype(np.uint32)
        res[f"{key}_rn_off"] = off
        res[f"{key}_out"] = np.array(outs)
        res[f"{key}_nout"] = np.array(nouts, dtype=np.int32)
        res[f"{key}_used"] = np.array(used, dtype=np.int64)
    np.savez_compressed(out, **res)


def _katspin(name, out):
    _kat(name, out, spin=True)


# Dose fixtures: name -> (case, spectrum or None, mono energy MeV, charge, histories)
DOSE = {
    "dose_water30": ("water30", "6mv", 1.25, 0, 2_000_000),
    "dose_slab64": ("slab64", "6mv", 1.25, 0, 2_000_000),
    "dose18_slab64": ("slab64", "18mv", 1.25, 0, 2_000_000),
    "dose_ctsmall": ("ctsmall", "6mv", 1.25, 0, 2_000_000),
    "dosee_water30": ("water30", None, 6.0, -1, 1_000_000),
    "dosep_water30": ("water30", None, 3.0, 1, 1_000_000),
    # photon splitting, nsplit = SPLIT (6th field)
    "dosesplit_water30": ("water30", "6mv", 1.25, 0, 1_000_000, SPLIT),
    "dosesplit_slab64": ("slab64", "6mv", 1.25, 0, 1_000_000, SPLIT),
    # the synthetic spin file (7th field): spin rejection and MS moment
    # corrections active; electrons of 6 MeV make the multiple scattering
    # the dominant physics
    "dosespin_slab64": ("slab64", "6mv", 1.25, 0, 2_000_000, 1, True),
    "doseespin_water30": ("water30", None, 6.0, -1, 1_000_000, 1, True),
}
SPIN_CASES = ["water30", "slab64", "ctsmall"]


def make_dose(fixture, nbatch=50, cores=8):
    """Reference CLI dose of one DOSE entry (voxels above 5 % of the max)."""
    from oracle.ref import run_cli
    name, spectrum, mono, charge, ncase = DOSE[fixture][:5]
    nsplit = DOSE[fixture][5] if len(DOSE[fixture]) > 5 else 1
    spin = DOSE[fixture][6] if len(DOSE[fixture]) > 6 else False
    A.require_assets()
    c = CASES[name]
    ph = c["phantom"]()
    pf = WORK / f"{name}.egsphant"
    if not pf.exists():
        A.write_egsphant(pf, ph)
    run = A.default_run(pf, spectrum=spectrum, ncase=ncase, nbatch=nbatch, collimator=c["collimator"],
                        mono_energy=mono, charge=charge)
    run.nsplit = nsplit
    if spin:
        run.data_folder = str(A.stage_spin_variant()) + "/"
    base = WORK / f"{fixture}_{ncase}"
    A.write_inp(base, run)
    loop_s, _ = run_cli(base, f"golden_{fixture}", cores=cores)
    dose, unc, _ = A.read_3ddose(A.ASSETS / "out" / f"golden_{fixture}.3ddose")
    keep = np.flatnonzero(dose.ravel() > 0.05 * dose.max())
    np.savez_compressed(HERE / f"{fixture}.npz", idx=keep.astype(np.int32), dose=dose.ravel()[keep],
                        unc=unc.ravel()[keep].astype(np.float32), shape=np.array(dose.shape), dmax=dose.max(),
                        ncase=ncase, nbatch=nbatch, loop_seconds=loop_s, cores=cores,
                        spectrum=str(spectrum or ""), mono_energy=mono, charge=charge, nsplit=nsplit,
                        spin_data="data_spin" if spin else "data")


GAMMA_HIST = {"water30": 100_000_000, "slab64": 400_000_000}


def make_gamma(name, nbatch=100, cores=8):
    """High-statistics reference dose for the gamma comparison."""
    from oracle.ref import run_cli
    ncase = GAMMA_HIST[name]
    base, ph = case_inp(name, ncase=ncase, nbatch=nbatch)
    loop_s, _ = run_cli(base, f"gamma_{name}", cores=cores, timeout=6 * 3600)
    dose, unc, _ = A.read_3ddose(A.ASSETS / "out" / f"gamma_{name}.3ddose")
    keep = np.flatnonzero(dose.ravel() > 0.02 * dose.max())
    np.savez_compressed(HERE / f"gamma_{name}.npz", idx=keep.astype(np.int32), dose=dose.ravel()[keep],
                        unc=unc.ravel()[keep].astype(np.float32), shape=np.array(dose.shape), dmax=dose.max(),
                        ncase=ncase, nbatch=nbatch, loop_seconds=loop_s, cores=cores)


# Full-size CT-like phantoms of the benchmark workloads: name -> (phantom,
# spectrum, histories, batches).  One reference CLI run each serves the
# z-test (its batch uncertainty) and the gamma test (its dose); the fixture
# keeps the voxels above 10 % of the maximum, dose as float32.
BIG = {
    # 128x128x96 x 0.3 cm, one 10x10 cm2 6 MV-like beam
    "ct128": (lambda: A.ct_phantom(128, 128, 96, 0.3, seed=1234), "6mv", 250_000_000, 50),
    # 256x256x160 x 0.2 cm, one 10x10 cm2 18 MV-like beam (pair/triplet production)
    "ct256": (A.ct_phantom_large, "18mv", 120_000_000, 40),
}


def make_big(name, cores=8):
    """Reference CLI dose of a BIG case -> refbig_<name>.npz."""
    from oracle.ref import run_cli
    mk, spectrum, ncase, nbatch = BIG[name]
    A.require_assets()
    ph = mk()
    pf = WORK / f"{name}.egsphant"
    if not pf.exists():
        A.write_egsphant(pf, ph)
    run = A.default_run(pf, spectrum=spectrum, ncase=ncase, nbatch=nbatch, collimator=(-5, 5, -5, 5))
    base = WORK / f"refbig_{name}_{ncase}"
    A.write_inp(base, run)
    loop_s, _ = run_cli(base, f"refbig_{name}", cores=cores, timeout=12 * 3600)
    dose, unc, _ = A.read_3ddose(A.ASSETS / "out" / f"refbig_{name}.3ddose")
    keep = np.flatnonzero(dose.ravel() > 0.1 * dose.max())
    np.savez_compressed(HERE / f"refbig_{name}.npz", idx=keep.astype(np.int32),
                        dose=dose.ravel()[keep].astype(np.float32), unc=unc.ravel()[keep].astype(np.float32),
                        shape=np.array(dose.shape), dmax=dose.max(), ncase=ncase, nbatch=nbatch,
                        loop_seconds=loop_s, cores=cores, spectrum=spectrum, collimator=np.array([-5, 5, -5, 5.0]))


# high-statistics reference doses of the BIG cases for the gamma test
GAMMA_BIG = {"ct128": (1_000_000_000, 100)}


def make_gamma_big(name, cores=8):
    """Reference CLI dose of a BIG case at GAMMA_BIG's histories ->
    gammabig_<name>.npz (voxels above 10 % of the maximum, float32)."""
    from oracle.ref import run_cli
    mk, spectrum, _, _ = BIG[name]
    ncase, nbatch = GAMMA_BIG[name]
    A.require_assets()
    pf = WORK / f"{name}.egsphant"
    if not pf.exists():
        A.write_egsphant(pf, mk())
    run = A.default_run(pf, spectrum=spectrum, ncase=ncase, nbatch=nbatch, collimator=(-5, 5, -5, 5))
    base = WORK / f"gammabig_{name}_{ncase}"
    A.write_inp(base, run)
    loop_s, _ = run_cli(base, f"gammabig_{name}", cores=cores, timeout=12 * 3600)
    dose, unc, _ = A.read_3ddose(A.ASSETS / "out" / f"gammabig_{name}.3ddose")
    keep = np.flatnonzero(dose.ravel() > 0.1 * dose.max())
    np.savez_compressed(HERE / f"gammabig_{name}.npz", idx=keep.astype(np.int32),
                        dose=dose.ravel()[keep].astype(np.float32), unc=unc.ravel()[keep].astype(np.float32),
                        shape=np.array(dose.shape), dmax=dose.max(), ncase=ncase, nbatch=nbatch,
                        loop_seconds=loop_s, cores=cores, spectrum=spectrum, collimator=np.array([-5, 5, -5, 5.0]))


DIJ = dict(gantry=[0.0, 90.0], bixel=1.0, field=(2.0, 2.0), nhist=100000, nbatch=10, rel=1e-4)


def make_dij(gaussian=False):
    """matRad D_ij of the ctsmall phantom from the unmodified MEX entry, one
    call per beamlet (each call starts its sums at zero, so V is the
    beamlet's own variance of the mean).  gaussian: the Gaussian focal spot
    (sourceGeometry 'gaussian', width 0.2123 cm) -> dijg_ctsmall.npz."""
    from oracle.ref import matrad_dij
    from ompmc_b200.engine import bixel_grid
    ph = CASES["ctsmall"]["phantom"]()
    bl = bixel_grid(ph, DIJ["gantry"], bixel=DIJ["bixel"], field=DIJ["field"])
    spec = A.ASSETS / "spectra" / "6mv.spectrum"
    cols, nnz_full = [], []
    for i in range(len(bl["corner"])):
        one = dict(bl, corner=bl["corner"][i:i + 1], side1=bl["side1"][i:i + 1], side2=bl["side2"][i:i + 1],
                   ibeam=bl["ibeam"][i:i + 1])
        jc, ir, pr, var = matrad_dij(ph, one, DIJ["nhist"], DIJ["nbatch"], seeds=(97, 33 + i),
                                     rel_threshold=DIJ["rel"], spectrum_file=str(spec), gaussian=gaussian)
        nnz_full.append(len(pr))
        keep = pr > 0.01 * pr.max()          # the fixture keeps entries above 1 % of the column maximum
        cols.append((ir[keep], pr[keep], var[keep]))
    colptr = np.concatenate([[0], np.cumsum([len(c[0]) for c in cols])])
    np.savez_compressed(HERE / ("dijg_ctsmall.npz" if gaussian else "dij_ctsmall.npz"), colptr=colptr, rows=np.concatenate([c[0] for c in cols]).astype(np.int32),
                        vals=np.concatenate([c[1] for c in cols]), var=np.concatenate([c[2] for c in cols]),
                        src=bl["src"], corner=bl["corner"], side1=bl["side1"], side2=bl["side2"], ibeam=bl["ibeam"],
                        nhist=DIJ["nhist"], nbatch=DIJ["nbatch"], rel=DIJ["rel"], nnz_full=np.array(nnz_full),
                        gaussian=int(gaussian))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    ap.add_argument("--cores", type=int, default=8, help="host cores of the refbig_* reference runs")
    a = ap.parse_args()
    from oracle.ref import build
    build()
    A.require_assets()
    WORK.mkdir(parents=True, exist_ok=True)
    jobs = [("rays", n) for n in CASES] + [("replay", n) for n in CASES] + [("replaysplit", n) for n in CASES]
    jobs += [("replayspin", n) for n in SPIN_CASES]
    jobs += [("kat", "slab64"), ("kat", "ctsmall"), ("katspin", "slab64")]
    for what, name in jobs:
        fn = f"{what}_{name}"
        if a.only and a.only not in fn:
            continue
        print("generating", fn, flush=True)
        _in_subprocess(name, what, HERE / f"{fn}.npz")
    for fixture in DOSE:
        if a.only and a.only not in fixture:
            continue
        print("generating", fixture, flush=True)
        make_dose(fixture)
    for name in GAMMA_HIST:
        if a.only and a.only not in f"gamma_{name}":
            continue
        print("generating gamma reference", name, flush=True)
        make_gamma(name)
    for name in BIG:
        if a.only and a.only not in f"refbig_{name}":
            continue
        print("generating refbig", name, flush=True)
        make_big(name, cores=a.cores)
    for name in GAMMA_BIG:
        if a.only and a.only not in f"gammabig_{name}":
            continue
        print("generating gammabig", name, flush=True)
        make_gamma_big(name, cores=a.cores)
    if not a.only or a.only in "dij_ctsmall":
        print("generating dij_ctsmall", flush=True)
        make_dij()
    if not a.only or a.only in "dijg_ctsmall":
        print("generating dijg_ctsmall", flush=True)
        make_dij(gaussian=True)


if __name__ == "__main__":
    main()
