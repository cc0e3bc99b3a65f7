"""Python host mirror of the engine's C ABI (include/omcgpu.h).

Mirrors ompMC's two surfaces for the transport path:

* `dosxyz(inp_base, out_name)` is the omc_dosxyz program
  (ucodes/omc_dosxyz/omc_dosxyz.c:1072-1307): same `.inp` keys, writes the
  same `.3ddose` file;
* `ompmc_b200.matrad.matrad_dij(cubeRho, cubeMatIx, mcGeo, mcSrc, mcOpt)`
  is the matRad MEX entry (ucodes/omc_matrad/omc_matrad.c:1417-1789): same
  inputs (dicts in place of MATLAB structs), returns scipy CSC matrices D
  (and V); it runs on `Engine.run_beamlets` below.

Errors raise `OmcError` carrying the library's status and message (the
reference calls exit() or mexErrMsgIdAndTxt).  The library is loaded from the
package directory; there is no fallback when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libomcgpu.so"
CLI_PATH = PKG / "bin" / "omc_dosxyz"

PLAIN_FP64 = 0
EVENT_FP32 = 1
EVENT_FP64 = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_up = C.POINTER(C.c_uint32)


class OmcError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


class _Phantom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("xb", _dp), ("yb", _dp), ("zb", _dp), ("med", _ip), ("rho", _dp)]


class _Options(C.Structure):
    _fields_ = [("ecut", C.c_double), ("pcut", C.c_double), ("device", C.c_int),
                ("ref_compat", C.c_int), ("queue_capacity", C.c_int64), ("block", C.c_int),
                ("nsplit", C.c_int), ("profile", C.c_int), ("electron_tsteps", C.c_int),
                ("inflight", C.c_int64), ("tail_boost", C.c_int), ("electron_split", C.c_double),
                ("electron_chsteps", C.c_int), ("electron_interact_kernel", C.c_int),
                ("photon_woodcock", C.c_int), ("drain_particles", C.c_int64)]


class _Energy(C.Structure):
    _fields_ = [("charge", C.c_int), ("mono_energy", C.c_double), ("n", C.c_int),
                ("cdf1", _dp), ("cdf2", _dp)]


class _Beam(C.Structure):
    _fields_ = [("energy", _Energy), ("ssd", C.c_double), ("xinl", C.c_double),
                ("xinu", C.c_double), ("yinl", C.c_double), ("yinu", C.c_double)]


class _Beamlets(C.Structure):
    _fields_ = [("energy", _Energy), ("nbeams", C.c_int), ("nbixels", C.c_int),
                ("ibeam", _ip), ("src", _dp), ("corner", _dp), ("side1", _dp), ("side2", _dp),
                ("gaussian", C.c_int), ("gauss_width", C.c_double)]


_lib = None


def lib():
    """Load libomcgpu.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise OmcError(-2, f"{LIB_PATH} is not built; run `make -C {PKG}`")
    L = C.CDLL(str(LIB_PATH))
    sig = {
        "omc_status_string": ([C.c_int], C.c_char_p),
        "omc_last_error": ([], C.c_char_p),
        "omc_version": ([], C.c_int),
        "omc_tables_build": ([C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int,
                              C.POINTER(C.c_void_p)], C.c_int),
        "omc_tables_free": ([C.c_void_p], None),
        "omc_tables_get": ([C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p), _lp, C.POINTER(C.c_int)], C.c_int),
        "omc_tables_nmed": ([C.c_void_p], C.c_int),
        "omc_spectrum_load": ([C.c_char_p, _dp, _dp, C.POINTER(C.c_int)], C.c_int),
        "omc_options_default": ([C.POINTER(_Options)], None),
        "omc_engine_create": ([C.c_void_p, C.POINTER(_Phantom), C.POINTER(_Options), C.POINTER(C.c_void_p)], C.c_int),
        "omc_engine_destroy": ([C.c_void_p], C.c_int),
        "omc_engine_last_error": ([C.c_void_p], C.c_char_p),
        "omc_run_beam": ([C.c_void_p, C.POINTER(_Beam), C.c_int64, C.c_int, C.c_uint64, C.c_int, _dp, _dp, _dp],
                         C.c_int),
        "omc_run_beamlets": ([C.c_void_p, C.POINTER(_Beamlets), C.c_int64, C.c_int, C.c_double, C.c_uint64, C.c_int,
                              _lp, _ip, _dp, _dp, C.c_int64, _lp, _dp], C.c_int),
        "omc_dosxyz_run": ([C.c_char_p, C.c_char_p, C.c_int, C.c_int], C.c_int),
        "omc_profile_last": ([C.c_void_p, _dp, C.c_int], C.c_int),
        "omc_profile_trace": ([C.c_void_p, _dp, C.c_int], C.c_int),
        "omc_profile_drain": ([C.c_void_p, _dp, C.c_int], C.c_int),
        "omc_event_params": ([C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_int, C.c_double, C.c_int, C.c_int64],
                             C.c_int),
        "omc_run_beam_noalloc": ([C.c_void_p, C.POINTER(_Beam), C.c_int64, C.c_int, C.c_uint64, _dp, _dp, _dp],
                                 C.c_int),
        "omc_server_create": ([C.c_void_p, C.c_int64, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)], C.c_int),
        "omc_server_destroy": ([C.c_void_p], C.c_int),
        "omc_server_submit_beamlet": ([C.c_void_p, C.POINTER(_Beamlets), C.c_int, C.c_int64, C.c_int, C.c_double,
                                       C.c_uint64], C.c_int),
        "omc_server_submit_beam": ([C.c_void_p, C.POINTER(_Beam), C.c_int64, C.c_int, C.c_uint64], C.c_int),
        "omc_server_step": ([C.c_void_p, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "omc_server_poll": ([C.c_void_p, C.c_int, _dp], C.c_int),
        "omc_server_result_sparse": ([C.c_void_p, C.c_int, _ip, _dp, _dp, C.c_int64, _lp], C.c_int),
        "omc_server_result_dense": ([C.c_void_p, C.c_int, _dp, _dp], C.c_int),
        "omc_server_release": ([C.c_void_p, C.c_int], C.c_int),
        "omc_trace_rays": ([C.c_void_p, _dp, C.c_int, C.c_int, _dp, _ip, _ip, _ip, _dp], C.c_int),
        "omc_replay": ([C.c_void_p, _dp, C.c_int, _dp, _lp, C.c_int, _ip, _dp, _ip, _lp, _up], C.c_int),
        "omc_device_allocations": ([], C.c_int64),
        "omc_kat": ([C.c_void_p, C.c_int, _dp, _dp, C.c_int, _dp, _lp, _dp, _ip, _lp, _up], C.c_int),
        "omc_server_completed": ([C.c_void_p, _ip, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "omc_server_timer": ([C.c_void_p, C.c_int, _dp], C.c_int),
        "omc_server_stats": ([C.c_void_p, _dp, C.c_int], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name, None)
        if f is None:
            continue
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def device_allocations():
    """Device allocations the library has made in this process."""
    return int(lib().omc_device_allocations())


def _check(rc, eng=None):
    if rc != 0:
        L = lib()
        msg = (L.omc_engine_last_error(eng) if eng else L.omc_last_error()) or b""
        raise OmcError(rc, msg.decode(errors="replace") or L.omc_status_string(rc).decode())


def _p(a, t):
    return a.ctypes.data_as(t)


class Tables:
    """Physics tables for the named media (initMediaData, ompmc.c:5468)."""

    def __init__(self, pegs_file, pgs4form_file, data_folder, media):
        L = lib()
        self.media = list(media)
        arr = (C.c_char_p * len(media))(*[m.encode() for m in media])
        h = C.c_void_p()
        data_folder = str(data_folder)
        if not data_folder.endswith("/"):
            data_folder += "/"
        _check(L.omc_tables_build(str(pegs_file).encode(), str(pgs4form_file).encode(), data_folder.encode(),
                                  arr, len(media), C.byref(h)))
        self.h = h

    @classmethod
    def from_assets(cls, media, root=None, data="data"):
        """Tables from the staged assets; `data` names the data folder under
        the assets root (`data_spin`: the synthetic spin file's variant)."""
        from . import assets
        root = Path(root) if root else assets.require_assets()
        return cls(root / "pegs4" / "521icru.pegs4dat", root / "pegs4" / "pgs4form.dat", root / data, media)

    def get(self, name):
        L = lib()
        ptr = C.c_void_p()
        n = C.c_int64()
        is_int = C.c_int()
        _check(L.omc_tables_get(self.h, name.encode(), C.byref(ptr), C.byref(n), C.byref(is_int)))
        if n.value == 0:
            return np.zeros(0)
        t = _ip if is_int.value else _dp
        return np.ctypeslib.as_array(C.cast(ptr, t), shape=(n.value,)).copy()

    def close(self):
        if getattr(self, "h", None):
            lib().omc_tables_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_spectrum(path):
    """Inverse CDF of a `.spectrum` file (omc_dosxyz.c:368-510)."""
    c1 = np.zeros(1000)
    c2 = np.zeros(1000)
    n = C.c_int()
    _check(lib().omc_spectrum_load(str(path).encode(), _p(c1, _dp), _p(c2, _dp), C.byref(n)))
    return c1[:n.value], c2[:n.value]


class Engine:
    """Resident tables + phantom on one GPU."""

    def __init__(self, tables: Tables, phantom, ecut=0.7, pcut=0.01, device=0, ref_compat=True,
                 queue_capacity=0, block=0, profile=False, electron_tsteps=0, inflight=0, tail_boost=0,
                 electron_split=None, nsplit=1, electron_chsteps=None, electron_interact_kernel=None,
                 photon_woodcock=None, drain_particles=None):
        L = lib()
        self.tables = tables
        self.phantom = phantom
        self._xb = np.ascontiguousarray(phantom.xb, dtype=np.float64)
        self._yb = np.ascontiguousarray(phantom.yb, dtype=np.float64)
        self._zb = np.ascontiguousarray(phantom.zb, dtype=np.float64)
        self._med = np.ascontiguousarray(phantom.med, dtype=np.int32).ravel()
        self._rho = np.ascontiguousarray(phantom.rho, dtype=np.float64).ravel()
        nx, ny, nz = phantom.shape
        self.shape = (nz, ny, nx)
        P = _Phantom(nx, ny, nz, _p(self._xb, _dp), _p(self._yb, _dp), _p(self._zb, _dp),
                     _p(self._med, _ip), _p(self._rho, _dp))
        o = _Options()
        L.omc_options_default(C.byref(o))
        o.ecut, o.pcut, o.device = ecut, pcut, device
        o.ref_compat = 1 if ref_compat else 0
        o.queue_capacity = queue_capacity
        o.block = block
        o.profile = 1 if profile else 0
        o.nsplit = int(nsplit)
        o.electron_tsteps = electron_tsteps
        o.inflight = inflight
        o.tail_boost = tail_boost
        if electron_split is not None:
            o.electron_split = electron_split
        if electron_chsteps is not None:
            o.electron_chsteps = int(electron_chsteps)
        if electron_interact_kernel is not None:
            o.electron_interact_kernel = int(electron_interact_kernel)
        if photon_woodcock is not None:
            o.photon_woodcock = int(photon_woodcock)
        if drain_particles is not None:
            o.drain_particles = int(drain_particles)
        h = C.c_void_p()
        _check(L.omc_engine_create(tables.h, C.byref(P), C.byref(o), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().omc_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _energy(spectrum=None, mono_energy=1.25, charge=0, keep=None):
        e = _Energy()
        e.charge = charge
        e.mono_energy = mono_energy
        if spectrum is not None:
            c1, c2 = (np.ascontiguousarray(a, dtype=np.float64) for a in spectrum)
            keep += [c1, c2]
            e.n = len(c1)
            e.cdf1, e.cdf2 = _p(c1, _dp), _p(c2, _dp)
        return e

    def run_beam(self, ncase, nbatch=10, seed=1, mode=EVENT_FP32, spectrum=None, mono_energy=1.25, charge=0,
                 ssd=100.0, collimator=(-5.0, 5.0, -5.0, 5.0), out=None):
        """Dose (Gy per history) and relative uncertainty arrays [nz,ny,nx]
        plus a stats dict; the dosxyz beam source (omc_dosxyz.c:964-1068).
        `out`: optional (dose, unc) float64 arrays of nvox elements to write
        into (e.g. pinned host memory)."""
        keep = []
        b = _Beam()
        b.energy = self._energy(spectrum, mono_energy, charge, keep)
        b.ssd = ssd
        b.xinl, b.xinu, b.yinl, b.yinu = collimator
        n = int(np.prod(self.shape))
        if out is not None:
            dose, unc = out
            assert dose.dtype == np.float64 and unc.dtype == np.float64 and dose.size == n and unc.size == n
            assert dose.flags.c_contiguous and unc.flags.c_contiguous
        else:
            dose = np.zeros(n)
            unc = np.zeros(n)
        st = np.zeros(6)
        _check(lib().omc_run_beam(self.h, C.byref(b), int(ncase), int(nbatch), int(seed) & (2**64 - 1), mode,
                                  _p(dose, _dp), _p(unc, _dp), _p(st, _dp)), self.h)
        stats = dict(histories=st[0], seconds=st[1], launches=int(st[2]), edep=st[3], esrc=st[4],
                     flags=int(st[5]))
        return dose.reshape(self.shape), unc.reshape(self.shape), stats

    def run_beam_noalloc(self, ncase, nbatch=10, seed=1, spectrum=None, mono_energy=1.25, charge=0, ssd=100.0,
                         collimator=(-5.0, 5.0, -5.0, 5.0)):
        """run_beam in the plain FP64 form on the library's fixed device
        scratch: for callers that must not allocate device memory during the
        run (see omc_run_beam_noalloc in include/omcgpu.h; at most
        OMC_NOALLOC_MAX_VOXELS = 262144 voxels; concurrent calls race)."""
        keep = []
        b = _Beam()
        b.energy = self._energy(spectrum, mono_energy, charge, keep)
        b.ssd = ssd
        b.xinl, b.xinu, b.yinl, b.yinu = collimator
        n = int(np.prod(self.shape))
        dose = np.zeros(n)
        unc = np.zeros(n)
        st = np.zeros(6)
        _check(lib().omc_run_beam_noalloc(self.h, C.byref(b), int(ncase), int(nbatch), int(seed) & (2**64 - 1),
                                          _p(dose, _dp), _p(unc, _dp), _p(st, _dp)), self.h)
        stats = dict(histories=st[0], seconds=st[1], launches=int(st[2]), edep=st[3], esrc=st[4],
                     flags=int(st[5]))
        return dose.reshape(self.shape), unc.reshape(self.shape), stats

    def run_beamlets(self, beamlets: dict, nhist, nbatch=10, rel_threshold=1e-4, seed=1, mode=EVENT_FP32,
                     with_variance=True):
        """matRad D_ij columns (omc_matrad.c:1576-1720) as CSC arrays."""
        keep = []
        b = self._beamlets_struct(beamlets, keep)
        nb = b.nbixels
        cap = int(beamlets.get("cap", max(1, int(np.prod(self.shape)) * nb // 20 + 1024)))
        for _ in range(3):
            colptr = np.zeros(nb + 1, dtype=np.int64)
            rows = np.zeros(cap, dtype=np.int32)
            vals = np.zeros(cap)
            var = np.zeros(cap) if with_variance else None
            nnz = C.c_int64()
            st = np.zeros(6)
            rc = lib().omc_run_beamlets(self.h, C.byref(b), int(nhist), int(nbatch), float(rel_threshold),
                                        int(seed), mode, _p(colptr, _lp), _p(rows, _ip), _p(vals, _dp),
                                        _p(var, _dp) if var is not None else None, cap, C.byref(nnz),
                                        _p(st, _dp))
            if rc == -5 and nnz.value > cap:
                cap = nnz.value
                continue
            _check(rc, self.h)
            k = nnz.value
            stats = dict(histories=st[0], seconds=st[1], launches=int(st[2]), flags=int(st[5]))
            return colptr, rows[:k], vals[:k], (var[:k] if var is not None else None), stats
        raise OmcError(-5, "sparse capacity kept growing")

    @staticmethod
    def _beamlets_struct(bl, keep):
        b = _Beamlets()
        b.energy = Engine._energy(bl.get("spectrum"), bl.get("mono_energy", 1.25), bl.get("charge", 0), keep)
        ibeam = np.ascontiguousarray(bl["ibeam"], dtype=np.int32)
        src = np.ascontiguousarray(bl["src"], dtype=np.float64).reshape(-1, 3)
        corner = np.ascontiguousarray(bl["corner"], dtype=np.float64).reshape(-1, 3)
        s1 = np.ascontiguousarray(bl["side1"], dtype=np.float64).reshape(-1, 3)
        s2 = np.ascontiguousarray(bl["side2"], dtype=np.float64).reshape(-1, 3)
        keep += [ibeam, src, corner, s1, s2]
        b.nbeams, b.nbixels = len(src), len(corner)
        b.ibeam, b.src, b.corner = _p(ibeam, _ip), _p(src, _dp), _p(corner, _dp)
        b.side1, b.side2 = _p(s1, _dp), _p(s2, _dp)
        b.gaussian = 1 if bl.get("gaussian") else 0
        b.gauss_width = float(bl.get("gauss_width", 0.2123))
        return b

    def profile_last(self):
        """Per-kernel profile of the last profiled event-form run."""
        out = np.zeros(28)
        _check(lib().omc_profile_last(self.h, _p(out, _dp), 28), self.h)
        names = ["source", "photon", "electron", "plan"]
        keys = ["launches", "seconds", "particles", "steps", "cross", "dep", "atom"]
        return {names[k]: dict(zip(keys, out[k * 7:(k + 1) * 7])) for k in range(4)}

    # ------------------------------------------------ validation hooks
    def event_params(self, electron_tsteps=0, tail_boost=0, inflight=0, block=0, electron_split=-1.0,
                     electron_chsteps=-1, drain_particles=-2):
        """Event-form tuning parameters (0, or -1 for electron_split and
        electron_chsteps, -2 for drain_particles, keeps the current value)."""
        _check(lib().omc_event_params(self.h, int(electron_tsteps), int(tail_boost), int(inflight), int(block),
                                      float(electron_split), int(electron_chsteps), int(drain_particles)), self.h)

    def profile_drain(self):
        """The drain of the last profiled event-form run: device ms, the
        particles it started from, and its largest thread sub-history
        (events, events of its first particle, transport steps)."""
        out = np.zeros(5)
        _check(lib().omc_profile_drain(self.h, _p(out, _dp), 5), self.h)
        return {"ms": out[0], "particles": int(out[1]), "max_events": int(out[2]), "max_chain_events": int(out[3]),
                "max_steps": int(out[4])}

    def profile_trace(self):
        """Per-cycle trace of the last profiled event-form run: array of rows
        (injected, photons in, electrons in, source ms, photon ms, electron ms)."""
        n = lib().omc_profile_trace(self.h, None, 0)
        _check(min(n, 0), self.h)
        out = np.zeros(max(n, 1) * 6)
        lib().omc_profile_trace(self.h, _p(out, _dp), n)
        return out[:n * 6].reshape(n, 6)

    def trace_rays(self, rays, cap=512):
        """FP64 device howfar walk per ray (x,y,z,u,v,w,ir)."""
        rays = np.ascontiguousarray(rays, dtype=np.float64)
        nr = len(rays)
        us = np.zeros((nr, cap))
        irn = np.zeros((nr, cap), dtype=np.int32)
        idc = np.zeros((nr, cap), dtype=np.int32)
        nc = np.zeros(nr, dtype=np.int32)
        hn = np.zeros(nr)
        _check(lib().omc_trace_rays(self.h, _p(rays, _dp), nr, cap, _p(us, _dp), _p(irn, _ip), _p(idc, _ip),
                                    _p(nc, _ip), _p(hn, _dp)), self.h)
        return us, irn, idc, nc, hn

    KAT = dict(compton=0, photo=1, pair=2, rayleigh=3, moller=4, bhabha=5, brems=6, annih=7, rannih=8, msdist=9)

    def kat(self, which, q, rn, rn_off, extra=None):
        """One FP64 sampler per case on scripted streams (omc_kat): returns
        out[n, 4, 11], nout, used, flags."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        n = len(q)
        rn = np.ascontiguousarray(rn, dtype=np.float64)
        off = np.ascontiguousarray(rn_off, dtype=np.int64)
        ex = None if extra is None else np.ascontiguousarray(extra, dtype=np.float64)
        out = np.zeros((n, 4, 11))
        nout = np.zeros(n, dtype=np.int32)
        used = np.zeros(n, dtype=np.int64)
        flags = np.zeros(n, dtype=np.uint32)
        _check(lib().omc_kat(self.h, self.KAT[which] if isinstance(which, str) else int(which), _p(q, _dp),
                             None if ex is None else _p(ex, _dp), n, _p(rn, _dp), _p(off, _lp), _p(out, _dp),
                             _p(nout, _ip), _p(used, _lp), _p(flags, _up)), self.h)
        return out, nout, used, flags

    def replay(self, prim, rn, rn_off, dep_cap=2048):
        """FP64 histories on recorded uniform streams; per-history deposits."""
        prim = np.ascontiguousarray(prim, dtype=np.float64)
        rn = np.ascontiguousarray(rn, dtype=np.float64)
        rn_off = np.ascontiguousarray(rn_off, dtype=np.int64)
        nh = len(prim)
        dir_ = np.zeros((nh, dep_cap), dtype=np.int32)
        de = np.zeros((nh, dep_cap))
        nd = np.zeros(nh, dtype=np.int32)
        nu = np.zeros(nh, dtype=np.int64)
        fl = np.zeros(nh, dtype=np.uint32)
        _check(lib().omc_replay(self.h, _p(prim, _dp), nh, _p(rn, _dp), _p(rn_off, _lp), dep_cap, _p(dir_, _ip),
                                _p(de, _dp), _p(nd, _ip), _p(nu, _lp), _p(fl, _up)), self.h)
        return dir_, de, nd, nu, fl


def dosxyz(inp_base, out_name, mode=EVENT_FP32, verbose=False):
    """The omc_dosxyz program: `<inp_base>.inp` in, `.3ddose` out."""
    _check(lib().omc_dosxyz_run(str(inp_base).encode(), str(out_name).encode(), mode, 1 if verbose else 0))


class Server:
    """Continuous batching of beamlet / beam requests on one engine
    (omc_server_* in include/omcgpu.h): requests are admitted while their
    tallies fit `mem_budget` bytes and share the engine's particle queues."""

    def __init__(self, engine: Engine, mem_budget=0, max_requests=0, seed=1):
        self.engine = engine
        h = C.c_void_p()
        _check(lib().omc_server_create(engine.h, int(mem_budget), int(max_requests), int(seed), C.byref(h)),
               engine.h)
        self.h = h
        self._keep = {}

    def beamlet_set(self, beamlets: dict):
        """Device-side description of a beamlet set; keep the returned
        object alive while its requests run."""
        keep = []
        b = Engine._beamlets_struct(beamlets, keep)
        self._keep[id(b)] = (b, keep)
        return b

    def submit_beamlet(self, bset, ibixel, nhist, nbatch=10, rel_threshold=1e-4, seed=0):
        rid = lib().omc_server_submit_beamlet(self.h, C.byref(bset), int(ibixel), int(nhist), int(nbatch),
                                              float(rel_threshold), int(seed))
        if rid < 0:
            _check(rid, self.engine.h)
        return rid

    def submit_beam(self, ncase, nbatch=10, spectrum=None, mono_energy=1.25, charge=0, ssd=100.0,
                    collimator=(-5.0, 5.0, -5.0, 5.0), seed=0):
        keep = []
        b = _Beam()
        b.energy = Engine._energy(spectrum, mono_energy, charge, keep)
        b.ssd = ssd
        b.xinl, b.xinu, b.yinl, b.yinu = collimator
        rid = lib().omc_server_submit_beam(self.h, C.byref(b), int(ncase), int(nbatch), int(seed))
        if rid < 0:
            _check(rid, self.engine.h)
        return rid

    def step(self, cycles=8):
        active = C.c_int()
        _check(lib().omc_server_step(self.h, int(cycles), C.byref(active)), self.engine.h)
        return active.value

    def poll(self, rid):
        lat = C.c_double()
        rc = lib().omc_server_poll(self.h, int(rid), C.byref(lat))
        if rc == -14:
            return None
        _check(rc, self.engine.h)
        return lat.value

    def result_sparse(self, rid):
        nnz = C.c_int64()
        lib().omc_server_result_sparse(self.h, int(rid), None, None, None, 0, C.byref(nnz))
        n = nnz.value
        rows = np.zeros(max(n, 1), dtype=np.int32)
        vals = np.zeros(max(n, 1))
        var = np.zeros(max(n, 1))
        _check(lib().omc_server_result_sparse(self.h, int(rid), _p(rows, _ip), _p(vals, _dp), _p(var, _dp), n,
                                              C.byref(nnz)), self.engine.h)
        return rows[:n], vals[:n], var[:n]

    def result_dense(self, rid):
        n = int(np.prod(self.engine.shape))
        dose = np.zeros(n)
        unc = np.zeros(n)
        _check(lib().omc_server_result_dense(self.h, int(rid), _p(dose, _dp), _p(unc, _dp)), self.engine.h)
        return dose.reshape(self.engine.shape), unc.reshape(self.engine.shape)

    def release(self, rid):
        _check(lib().omc_server_release(self.h, int(rid)), self.engine.h)

    def completed(self, cap=4096):
        """Ids of the requests finished since the previous call, in order."""
        ids = np.zeros(cap, dtype=np.int32)
        n = C.c_int()
        _check(lib().omc_server_completed(self.h, _p(ids, _ip), int(cap), C.byref(n)), self.engine.h)
        return ids[:n.value].tolist()

    def stats(self):
        """Cycles, drains, kernel launches and finished requests so far."""
        out = np.zeros(4)
        _check(lib().omc_server_stats(self.h, _p(out, _dp), 4), self.engine.h)
        return dict(cycles=int(out[0]), drains=int(out[1]), launches=int(out[2]), finished=int(out[3]))

    def timer_start(self):
        """Mark the start of a device-timed span on the server's stream."""
        _check(lib().omc_server_timer(self.h, 0, None), self.engine.h)

    def timer_stop(self):
        """Device milliseconds since timer_start (waits for the stream)."""
        ms = C.c_double()
        _check(lib().omc_server_timer(self.h, 1, C.byref(ms)), self.engine.h)
        return ms.value

    def close(self):
        if getattr(self, "h", None):
            lib().omc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bixel_grid(phantom, gantry_deg, bixel=0.5, field=(5.0, 5.0), sad=100.0, iso=None):
    """matRad-style beamlets of coplanar beams rotating about the z axis:
    for each gantry angle a source point at distance `sad` from the
    isocentre and a grid of `bixel`-sized squares (side1, side2) in the plane
    through the isocentre perpendicular to the beam.  Returns the dict
    accepted by Engine.run_beamlets / Server.beamlet_set."""
    xb, yb, zb = phantom.xb, phantom.yb, phantom.zb
    if iso is None:
        iso = np.array([(xb[0] + xb[-1]) / 2, (yb[0] + yb[-1]) / 2, (zb[0] + zb[-1]) / 2])
    src, corner, s1, s2, ibeam = [], [], [], [], []
    nu = int(round(field[0] / bixel))
    nv = int(round(field[1] / bixel))
    for b, g in enumerate(gantry_deg):
        t = np.deg2rad(g)
        d = np.array([np.sin(t), -np.cos(t), 0.0])      # beam direction (source -> iso)
        src.append(iso - sad * d)
        e1 = np.array([np.cos(t), np.sin(t), 0.0]) * bixel
        e2 = np.array([0.0, 0.0, 1.0]) * bixel
        for i in range(nu):
            for j in range(nv):
                c = iso + (i - nu / 2) * e1 + (j - nv / 2) * e2
                corner.append(c)
                s1.append(e1)
                s2.append(e2)
                ibeam.append(b)
    return dict(src=np.array(src), corner=np.array(corner), side1=np.array(s1), side2=np.array(s2),
                ibeam=np.array(ibeam, dtype=np.int32))
