"""ctypes view of the oracle harness (oracle/harness.c) around the unmodified
ompMC reference built by oracle/Makefile into oracle/_ref/.

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.

The reference keeps all state in process globals (ompmc.h:114-435), so one
process holds one configuration: `Reference.open(inp_base)` initialises it
once and later calls with another `.inp` raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
LIB = REF_DIR / "libompmc_ref.so"
CLI = REF_DIR / "omc_dosxyz_ref"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)


def build(reference_root="/root/reference"):
    """Build oracle/_ref from an ompMC checkout (no-op when up to date)."""
    if not Path(reference_root).is_dir():
        if LIB.exists() and CLI.exists():
            return
        raise FileNotFoundError("oracle/_ref is not built and no ompMC checkout is present")
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={reference_root}"], check=True)


def available():
    return LIB.exists() and CLI.exists()


def _p(a, t):
    return a.ctypes.data_as(t)


class Reference:
    _inst = None

    def __init__(self):
        self.lib = C.CDLL(str(LIB))
        L = self.lib
        L.h_init.argtypes = [C.c_char_p]
        L.h_table.argtypes = [C.c_char_p, _lp]
        L.h_table.restype = C.c_void_p
        L.h_howfar.argtypes = [C.c_double] * 6 + [C.c_int, C.c_double, _dp, _ip, _ip]
        L.h_hownear.argtypes = [C.c_double] * 3 + [C.c_int]
        L.h_hownear.restype = C.c_double
        L.h_walk.argtypes = [C.c_double] * 6 + [C.c_int, C.c_int, _dp, _ip, _ip]
        L.h_source.argtypes = [_dp]
        L.h_run.argtypes = [C.c_int, _dp, _dp, C.c_long, _lp, _ip, _dp, C.c_long, _lp]
        L.h_replay.argtypes = [_dp, _dp, C.c_long, _ip, _dp, C.c_long, _lp]
        L.h_replay.restype = C.c_long
        L.h_sampler.argtypes = [C.c_int, _dp, _dp, C.c_long, _lp, _dp]
        L.h_msdist.argtypes = [_dp, C.c_double, C.c_double, _dp, C.c_long, _lp, _dp]
        L.h_msdist.restype = C.c_double
        L.h_spin_scalars.argtypes = [_dp]
        self.inp = None

    @classmethod
    def open(cls, inp_base):
        """Initialise the reference on `<inp_base>.inp` (once per process)."""
        if cls._inst is None:
            cls._inst = Reference()
        r = cls._inst
        inp_base = str(inp_base)
        if r.inp is None:
            r.lib.h_init(inp_base.encode())
            r.inp = inp_base
        elif r.inp != inp_base:
            raise RuntimeError(f"reference already initialised on {r.inp}")
        return r

    # ------------------------------------------------------------ tables
    INT_TABLES = {"i_array", "ims", "sig_ismonotone", "meke", "region_med"}

    def table(self, name):
        n = C.c_long(0)
        ptr = self.lib.h_table(name.encode(), C.byref(n))
        if not ptr:
            raise KeyError(name)
        if name in self.INT_TABLES:
            return np.ctypeslib.as_array(C.cast(ptr, _ip), shape=(n.value,)).copy()
        return np.ctypeslib.as_array(C.cast(ptr, _dp), shape=(n.value,)).copy()

    def spin_scalars(self):
        out = np.zeros(7)
        self.lib.h_spin_scalars(_p(out, _dp))
        return dict(zip(["b2spin_min", "dbeta2i", "espml", "dleneri", "dqq1i",
                         "dllambi", "dqmsi"], out))

    # ---------------------------------------------------------- geometry
    def howfar(self, x, y, z, u, v, w, ir, ustep):
        us = C.c_double()
        irn = C.c_int()
        idisc = C.c_int()
        self.lib.h_howfar(x, y, z, u, v, w, int(ir), ustep, C.byref(us), C.byref(irn), C.byref(idisc))
        return us.value, irn.value, idisc.value

    def hownear(self, x, y, z, ir):
        return self.lib.h_hownear(x, y, z, int(ir))

    def walk(self, x, y, z, u, v, w, ir, cap=4096):
        us = np.zeros(cap)
        irn = np.zeros(cap, dtype=np.int32)
        idisc = np.zeros(cap, dtype=np.int32)
        n = self.lib.h_walk(x, y, z, u, v, w, int(ir), cap, _p(us, _dp), _p(irn, _ip), _p(idisc, _ip))
        return us[:n], irn[:n], idisc[:n]

    # --------------------------------------------------------- histories
    def source(self):
        q = np.zeros(11)
        self.lib.h_source(_p(q, _dp))
        return q

    def run(self, nhist, rn_cap=None, dep_cap=None):
        """Run `nhist` histories with RANMAR; returns primaries[nhist,11],
        per-history random streams and deposit sequences (ir, e)."""
        rn_cap = rn_cap or nhist * 4000
        dep_cap = dep_cap or nhist * 400
        prim = np.zeros((nhist, 11))
        rn = np.zeros(rn_cap)
        rn_off = np.zeros(nhist + 1, dtype=np.int64)
        dir_ = np.zeros(dep_cap, dtype=np.int32)
        de = np.zeros(dep_cap)
        d_off = np.zeros(nhist + 1, dtype=np.int64)
        rc = self.lib.h_run(nhist, _p(prim, _dp), _p(rn, _dp), rn_cap, _p(rn_off, _lp),
                            _p(dir_, _ip), _p(de, _dp), dep_cap, _p(d_off, _lp))
        if rc != 0:
            raise RuntimeError("oracle buffers overflowed; raise rn_cap/dep_cap")
        return dict(prim=prim, rn=rn[:rn_off[-1]].copy(), rn_off=rn_off,
                    dep_ir=dir_[:d_off[-1]].copy(), dep_e=de[:d_off[-1]].copy(), d_off=d_off)

    def replay(self, q, rn, dep_cap=100000):
        q = np.ascontiguousarray(q, dtype=np.float64)
        rn = np.ascontiguousarray(rn, dtype=np.float64)
        dir_ = np.zeros(dep_cap, dtype=np.int32)
        de = np.zeros(dep_cap)
        nd = C.c_long()
        used = self.lib.h_replay(_p(q, _dp), _p(rn, _dp), len(rn), _p(dir_, _ip), _p(de, _dp),
                                 dep_cap, C.byref(nd))
        return used, dir_[:nd.value].copy(), de[:nd.value].copy()

    SAMPLERS = dict(compton=0, photo=1, pair=2, rayleigh=3, moller=4, bhabha=5,
                    brems=6, annih=7, rannih=8)

    def sampler(self, name, q, rn):
        q = np.ascontiguousarray(q, dtype=np.float64)
        rn = np.ascontiguousarray(rn, dtype=np.float64)
        out = np.zeros((4, 11))
        used = C.c_long()
        n = self.lib.h_sampler(self.SAMPLERS[name], _p(q, _dp), _p(rn, _dp), len(rn),
                               C.byref(used), _p(out, _dp))
        return used.value, out[:n].copy()

    def msdist(self, q, de, tustep, rn):
        q = np.ascontiguousarray(q, dtype=np.float64)
        rn = np.ascontiguousarray(rn, dtype=np.float64)
        fin = np.zeros(6)
        used = C.c_long()
        ustep = self.lib.h_msdist(_p(q, _dp), de, tustep, _p(rn, _dp), len(rn), C.byref(used), _p(fin, _dp))
        return ustep, used.value, fin


MATRAD_LIB = REF_DIR / "libompmc_matrad_ref.so"


_mex_libs = {}


def matrad_dij(phantom, beamlets, nhist, nbatch=10, seeds=(97, 33), ecut=0.7, pcut=0.01, rel_threshold=1e-4,
               spectrum_file="", assets_root=None, gaussian=False, gauss_width=0.2123, cap=None, lib=None):
    """One call of the unmodified matRad MEX entry (omc_matrad.c:1417) through
    the mex.h shim.  `beamlets` is the dict of ompmc_b200.engine.bixel_grid
    (0-based ibeam).  Returns (colptr, rows, vals, var) of D and V.  `lib`:
    another build of the shim harness linked with a different mexFunction
    (the tests use it to drive this project's MEX entry the same way)."""
    from ompmc_b200 import assets as A
    root = Path(assets_root) if assets_root else A.require_assets()
    path = str(lib or MATRAD_LIB)
    if path not in _mex_libs:
        L = C.CDLL(path)
        L.hm_dij.restype = C.c_long
        L.hm_last_error.restype = C.c_char_p
        _mex_libs[path] = L
    L = _mex_libs[path]
    nx, ny, nz = phantom.shape
    rho = np.ascontiguousarray(phantom.rho, dtype=np.float64).ravel()
    mat = np.ascontiguousarray(phantom.med, dtype=np.int32).ravel()
    names = (C.c_char_p * len(phantom.media))(*[m.encode() for m in phantom.media])
    xb, yb, zb = (np.ascontiguousarray(b, dtype=np.float64) for b in (phantom.xb, phantom.yb, phantom.zb))
    ib = np.asarray(beamlets["ibeam"], dtype=np.float64) + 1.0
    src = np.ascontiguousarray(beamlets["src"], dtype=np.float64)
    cor = np.ascontiguousarray(beamlets["corner"], dtype=np.float64)
    s1 = np.ascontiguousarray(beamlets["side1"], dtype=np.float64)
    s2 = np.ascontiguousarray(beamlets["side2"], dtype=np.float64)
    nbix, nbeams = len(cor), len(src)
    cap = cap or max(1024, nx * ny * nz * nbix // 4)
    jc = np.zeros(nbix + 1, dtype=np.int64)
    ir = np.zeros(cap, dtype=np.int64)
    pr = np.zeros(cap)
    var = np.zeros(cap)
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))
    n = L.hm_dij(C.c_int(nx), C.c_int(ny), C.c_int(nz), P(rho, C.c_double), P(mat, C.c_int32),
                 C.c_int(len(phantom.media)), names, P(xb, C.c_double), P(yb, C.c_double), P(zb, C.c_double),
                 C.c_int(nbix), C.c_int(nbeams), P(ib, C.c_double), P(src, C.c_double), P(cor, C.c_double),
                 P(s1, C.c_double), P(s2, C.c_double), C.c_double(nhist), C.c_double(nbatch),
                 C.c_double(seeds[0]), C.c_double(seeds[1]), C.c_double(ecut), C.c_double(pcut),
                 C.c_double(rel_threshold), str(spectrum_file).encode(),
                 str(root / "pegs4" / "521icru.pegs4dat").encode(), str(root / "pegs4" / "pgs4form.dat").encode(),
                 (str(root / "data") + "/").encode(), (str(root / "out") + "/").encode(), C.c_int(int(gaussian)),
                 C.c_double(gauss_width), P(jc, C.c_long), P(ir, C.c_long), P(pr, C.c_double), P(var, C.c_double),
                 C.c_long(cap))
    if n < 0:
        raise RuntimeError(f"matRad reference failed ({n}): {L.hm_last_error().decode(errors='replace')}")
    return jc, ir[:n].copy(), pr[:n].copy(), var[:n].copy()


def run_cli(inp_base, out_name, cores=None, timeout=3600):
    """Run the reference CLI on `<inp_base>.inp`; returns (seconds of the
    batch loop as the CLI reports it, path of the .3ddose).  `cores` pins
    the process with taskset (omc_dosxyz.c:1159-1161 sizes its thread pool
    with omp_get_num_procs, which follows the affinity mask)."""
    cmd = [str(CLI), "-i", str(inp_base), "-o", out_name]
    if cores:
        cmd = ["taskset", "-c", f"0-{cores - 1}"] + cmd
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(p.stdout[-2000:] + p.stderr[-2000:])
    times = [float(l.split(":")[1].split()[0]) for l in p.stdout.splitlines()
             if l.startswith("Execution time up to this point")]
    loop = times[1] - times[0] if len(times) >= 2 else float("nan")
    return loop, p.stdout
