"""Input assets for the dose engine: physics data staging, the stand-in spin
table, synthetic spectra and phantoms, and the ompMC text formats.

ompMC reads its physics data from files named by `.inp` keys
(`pegs file`, `pgs4form file`, `data folder`; ompMC `src/ompmc.c:472-522`,
`:758-819`, `:3219-3298`, `:2394-2625`).  This module stages those files from
an ompMC checkout into `assets/` (git-ignored) and writes the one file the
upstream tree does not ship, `spinms.data`.

Stand-in spin table
-------------------
`data/spinms.data` is missing upstream, and ompMC exits without it
(`src/ompmc.c:2412-2415`).  `write_spin_standin` writes a file in the exact
binary layout `initSpinData` reads (`src/ompmc.c:2424-2625`):

* record size 1104 bytes (276 float32); record 0 holds a 32-byte version
  string, a 4-byte endianness tag, then float32 `espin_min, espin_max`
  (keV) and `b2spin_min, b2spin_max`;
* element Z, charge index q (0 = e-, 1 = e+) and energy index i (0..31)
  live in record `1 + (Z-1)*64 + 32*q + i`; each holds float32
  `dum1, dum2, dum3, aux_o`, float32 `fmax[16]`, then 512 uint16 at int16
  offset 40: the rejection surface `spin_rej[q][j][k]` as fractions of
  `fmax[j]`.

The stand-in is neutral: every surface point is 65535 and `fmax = 1`, so the
Mott/spin rejection function is identically 1 ("spin-off" physics);
`dum1 = dum3 = 1` makes the first-moment correction 1 for a single element;
`dum2` is set to the screened-Rutherford q2/q1 ratio `gamma(eta)` of the
element itself so the second-moment correction is 1 for a single element;
`aux_o = 1.13` (screening-parameter correction).  Energy grid: 1 keV to
100 keV (log), then beta^2 from beta^2(100 keV) to 0.999.  Both the reference
oracle and this engine read the same file, so parity is exact in definition;
the physics is no longer EGSnrc-validated.
"""
from __future__ import annotations

import math
import os
import shutil
import struct
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

RM = 0.5109989461  # MeV, electron rest energy (ompMC src/ompmc.h:47)

REPO = Path(__file__).resolve().parent.parent
ASSETS = REPO / "assets"

# Spin stand-in parameters (documented in the module docstring).
SPIN_ESPIN_MIN_KEV = 1.0
SPIN_ESPIN_MAX_KEV = 100.0
SPIN_B2_MAX = 0.999
SPIN_AUX_O = 1.13
SPIN_ZMAX = 100
_MXE_SPIN = 15
_MXQ_SPIN = 15
_MXU_SPIN = 31
_REC_FLOATS = 276


def _spin_energy_grid(espin_min, espin_max, b2min, b2max):
    """Energy grid (keV) implied by the file header, as `initSpinData`
    rebuilds it (ompMC src/ompmc.c:2476-2501)."""
    nener = _MXE_SPIN
    earray = np.zeros(2 * nener + 2)
    dloge = math.log(espin_max / espin_min) / nener
    eloge = math.log(espin_min)
    earray[0] = espin_min
    for i in range(1, nener + 1):
        eloge += dloge
        earray[i] = math.exp(eloge)
    dbeta2 = (b2max - b2min) / nener
    beta2 = b2min
    earray[nener + 1] = espin_max
    for i in range(nener + 2, 2 * nener + 2):
        beta2 += dbeta2
        earray[i] = RM * 1000.0 * (1.0 / math.sqrt(1.0 - beta2) - 1.0) if beta2 < 0.999 else 50585.1
    return earray


def _gamma_of_eta(eta):
    """q2/q1 of the screened Rutherford cross section at screening eta."""
    l = math.log(1.0 + 1.0 / eta)
    return 3.0 * (1.0 + eta) * (l * (1.0 + 2.0 * eta) - 2.0) / (l * (1.0 + eta) - 1.0)


def write_spin_standin(path, zmax=SPIN_ZMAX):
    """Write the neutral stand-in spin file described in the module docstring."""
    espin_min, espin_max = SPIN_ESPIN_MIN_KEV, SPIN_ESPIN_MAX_KEV
    tau_max = espin_max / (1000.0 * RM)
    b2min = tau_max * (tau_max + 2.0) / (tau_max + 1.0) ** 2
    b2max = SPIN_B2_MAX
    earray = _spin_energy_grid(espin_min, espin_max, np.float32(b2min), np.float32(b2max))
    nrec = 1 + zmax * 64
    buf = bytearray(nrec * _REC_FLOATS * 4)
    hdr = b"stand-in neutral spin data v1".ljust(32, b" ") + b"LITL"
    buf[0:36] = hdr
    struct.pack_into("<4f", buf, 36, espin_min, espin_max, b2min, b2max)
    surface = np.full(512, 65535, dtype=np.uint16).tobytes()
    fmax = struct.pack("<16f", *([1.0] * 16))
    tf = 137.03604 * 0.88534138
    for z in range(1, zmax + 1):
        z23 = z ** (2.0 / 3.0)
        for q in range(2):
            for i in range(2 * _MXE_SPIN + 2):
                tau = earray[i] / (1000.0 * RM)
                eta = z23 / (tf * tf) * SPIN_AUX_O / 4.0 / tau / (tau + 2.0)
                dum2 = _gamma_of_eta(eta)
                rec = 1 + (z - 1) * 64 + 32 * q + i
                off = rec * _REC_FLOATS * 4
                struct.pack_into("<4f", buf, off, 1.0, dum2, 1.0, SPIN_AUX_O)
                buf[off + 16: off + 80] = fmax
                buf[off + 80: off + 80 + 1024] = surface
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "wb") as f:
        f.write(bytes(buf))
    return path


def write_spin_synthetic(path, seed=2024, zmax=SPIN_ZMAX):
    """Write a seeded, non-constant spin file in the same layout, to exercise
    the spin-dependent code paths (Mott/spin rejection in the multiple
    scattering sampler, the first- and second-moment corrections of the MS
    step): it is test data, not physics.

    For element Z, charge q, energy index i and q-index j, the surface over
    the 32 u-nodes k is the smooth, strictly positive
        s(k) = 1 - a * (1 - cos(pi * k / 31)) / 2 * (1 + b * sin(pi * k / 11)),
    a in [0.1, 0.6] and b in [-0.15, 0.15] varying smoothly with (Z, q, i, j)
    plus a seeded random part; fmax[j] in [0.6, 1.4]; dum1, dum3 (first-moment
    factors) within 8 % of 1 and dum2 within 6 % of the neutral gamma(eta),
    so the q1 and q2 corrections differ from 1."""
    rng = np.random.default_rng(seed)
    espin_min, espin_max = SPIN_ESPIN_MIN_KEV, SPIN_ESPIN_MAX_KEV
    tau_max = espin_max / (1000.0 * RM)
    b2min = tau_max * (tau_max + 2.0) / (tau_max + 1.0) ** 2
    b2max = SPIN_B2_MAX
    earray = _spin_energy_grid(espin_min, espin_max, np.float32(b2min), np.float32(b2max))
    nrec = 1 + zmax * 64
    buf = bytearray(nrec * _REC_FLOATS * 4)
    hdr = b"stand-in synthetic spin data v1".ljust(32, b" ") + b"LITL"
    buf[0:36] = hdr
    struct.pack_into("<4f", buf, 36, espin_min, espin_max, b2min, b2max)
    tf = 137.03604 * 0.88534138
    k = np.arange(32)
    for z in range(1, zmax + 1):
        z23 = z ** (2.0 / 3.0)
        for q in range(2):
            for i in range(2 * _MXE_SPIN + 2):
                tau = earray[i] / (1000.0 * RM)
                eta = z23 / (tf * tf) * SPIN_AUX_O / 4.0 / tau / (tau + 2.0)
                ph = 0.37 * z + 1.3 * q + 0.21 * i
                dum1 = 1.0 + 0.05 * math.sin(ph) + 0.03 * (rng.random() - 0.5)
                dum3 = 1.0 + 0.04 * math.cos(0.5 * ph) + 0.03 * (rng.random() - 0.5)
                dum2 = _gamma_of_eta(eta) * (1.0 + 0.05 * math.sin(0.7 * ph + 0.4) + 0.02 * (rng.random() - 0.5))
                rec = 1 + (z - 1) * 64 + 32 * q + i
                off = rec * _REC_FLOATS * 4
                struct.pack_into("<4f", buf, off, dum1, dum2, dum3, SPIN_AUX_O)
                fmax = 0.6 + 0.8 * rng.random(16)
                buf[off + 16: off + 80] = struct.pack("<16f", *fmax)
                surf = np.zeros((16, 32))
                for j in range(16):
                    a = 0.35 + 0.25 * math.sin(0.11 * z + 0.9 * q + 0.17 * i + 0.29 * j) * 0.8 + 0.1 * rng.random()
                    a = min(max(a, 0.1), 0.6)
                    b = 0.15 * math.sin(0.3 * i + 0.7 * j + q)
                    surf[j] = 1.0 - a * (1.0 - np.cos(np.pi * k / 31.0)) / 2.0 * (1.0 + b * np.sin(np.pi * k / 11.0))
                u16 = np.clip(np.round(surf * 65535.0), 1, 65535).astype(np.uint16)
                buf[off + 80: off + 80 + 1024] = u16.tobytes()
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "wb") as f:
        f.write(bytes(buf))
    return path


def stage_spin_variant(root=ASSETS):
    """A second data folder, `data_spin/`, holding the same cross-section and
    multiple-scattering files and the synthetic spin file; returns it."""
    root = Path(root)
    src = require_assets(root) / "data"
    dst = root / "data_spin"
    if (dst / "spinms.data").exists() and all((dst / f).exists() for f in DATA_FILES):
        return dst
    dst.mkdir(parents=True, exist_ok=True)
    for f in DATA_FILES:
        shutil.copyfile(src / f, dst / f)
    write_spin_synthetic(dst / "spinms.data")
    return dst


# --------------------------------------------------------------------------
# Staging of the physics data shipped by ompMC
# --------------------------------------------------------------------------
DATA_FILES = ["xcom_photo.data", "xcom_rayleigh.data", "xcom_pair.data",
              "xcom_triplet.data", "msnew.data"]
PEGS_FILES = ["521icru.pegs4dat", "pgs4form.dat"]


def assets_ready(root=ASSETS):
    root = Path(root)
    need = [root / "data" / f for f in DATA_FILES + ["spinms.data"]]
    need += [root / "pegs4" / f for f in PEGS_FILES]
    return all(p.exists() for p in need)


def stage(reference_root=None, root=ASSETS, force=False):
    """Copy ompMC's physics data into `root` and write the stand-in spin file.

    `reference_root` is an ompMC checkout (default: the OMPMC_REFERENCE
    environment variable).  Returns the assets root.  Raises
    FileNotFoundError when neither the staged files nor an ompMC checkout
    are available.
    """
    root = Path(root)
    if assets_ready(root) and not force:
        return root
    if reference_root is None:
        reference_root = os.environ.get("OMPMC_REFERENCE", "")
    if not reference_root:
        raise FileNotFoundError(f"physics data not staged under {root}; pass an ompMC checkout "
                                "(stage(reference_root=...) or OMPMC_REFERENCE)")
    ref = Path(reference_root)
    if not (ref / "data").is_dir():
        raise FileNotFoundError(
            f"physics data not staged under {root} and no ompMC checkout at {ref}")
    (root / "data").mkdir(parents=True, exist_ok=True)
    (root / "pegs4").mkdir(parents=True, exist_ok=True)
    (root / "spectra").mkdir(parents=True, exist_ok=True)
    for f in DATA_FILES:
        shutil.copyfile(ref / "data" / f, root / "data" / f)
    for f in PEGS_FILES:
        shutil.copyfile(ref / "pegs4" / f, root / "pegs4" / f)
    for f in (ref / "spectra").glob("*.spectrum"):
        shutil.copyfile(f, root / "spectra" / f.name)
    write_spin_standin(root / "data" / "spinms.data")
    return root


def require_assets(root=ASSETS):
    """Return the assets root, staging it from an ompMC checkout if needed
    (its `out` folder, where runs write their outputs, is created)."""
    root = Path(root) if assets_ready(root) else stage(root=root)
    (root / "out").mkdir(parents=True, exist_ok=True)
    return root


# --------------------------------------------------------------------------
# Spectra
# --------------------------------------------------------------------------
def spectrum_bins(nbins, emin, emax, ecut_scale):
    """Equal-width bins with weights E^-0.5 exp(-E/scale) at the bin centres,
    normalised (counts/bin).  Returns (upper edges, weights, mean energy)."""
    edges = emin + (emax - emin) * np.arange(nbins + 1) / nbins
    centres = 0.5 * (edges[1:] + edges[:-1])
    w = centres ** -0.5 * np.exp(-centres / ecut_scale)
    w = w / w.sum()
    mean = float((w * centres).sum())
    return edges[1:], w, mean


SPECTRA = {
    # 6 MV-like: 24 bins 0.25..6.0 MeV, E^-0.5 exp(-E/2.0)
    "6mv": dict(nbins=24, emin=0.25, emax=6.0, scale=2.0),
    # 18 MV-like: 36 bins 0.25..18 MeV, E^-0.5 exp(-E/5.5)
    "18mv": dict(nbins=36, emin=0.25, emax=18.0, scale=5.5),
}


def write_spectrum(path, name="6mv"):
    """Write an ompMC `.spectrum` file (title; `nbins emin imode`; `E_upper w`
    lines; format read by omc_dosxyz.c:368-430)."""
    p = SPECTRA[name]
    upper, w, mean = spectrum_bins(p["nbins"], p["emin"], p["emax"], p["scale"])
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        f.write(f" {name} synthetic spectrum E^-0.5 exp(-E/{p['scale']}) mean {mean:.4f} MeV\n")
        f.write(f"   {p['nbins']} {p['emin']} 0\n")
        for e, wi in zip(upper, w):
            f.write(f"   {e:.6f} {wi:.9e}\n")
    return path


# --------------------------------------------------------------------------
# Phantoms
# --------------------------------------------------------------------------
@dataclass
class Phantom:
    """Rectilinear voxel phantom.  Arrays are indexed [k, j, i] (z, y, x),
    i.e. x fastest in memory, matching ompMC's region numbering
    `ir = 1 + i + j*nx + k*nx*ny` (omc_dosxyz.c:124-128)."""
    media: list
    xb: np.ndarray
    yb: np.ndarray
    zb: np.ndarray
    med: np.ndarray      # int32, 1-based medium index per voxel
    rho: np.ndarray      # float64 mass density per voxel
    name: str = "phantom"

    @property
    def shape(self):
        return (len(self.xb) - 1, len(self.yb) - 1, len(self.zb) - 1)

    @property
    def nvox(self):
        nx, ny, nz = self.shape
        return nx * ny * nz


def _grid(n, d, lo):
    """Boundaries rounded to the 6 decimals of the `.egsphant` text, so the
    arrays handed to the engine equal what a reader of the file gets."""
    return np.round(lo + d * np.arange(n + 1, dtype=np.float64), 6)


def water_cube(n=30, d=1.0):
    """Homogeneous water, x,y in [-n*d/2, n*d/2], z in [0, n*d]."""
    xb = _grid(n, d, -n * d / 2)
    zb = _grid(n, d, 0.0)
    med = np.ones((n, n, n), dtype=np.int32)
    rho = np.ones((n, n, n), dtype=np.float64)
    return Phantom(["H2O521ICRU"], xb, xb.copy(), zb, med, rho, name=f"water{n}")


def slab_phantom(n=64, d=0.25):
    """Water 0-3 cm, lung (0.26) 3-8 cm, bone (1.85) 8-10 cm, water to the end."""
    xb = _grid(n, d, -n * d / 2)
    zb = _grid(n, d, 0.0)
    zc = 0.5 * (zb[1:] + zb[:-1])
    medz = np.ones(n, dtype=np.int32)
    rhoz = np.ones(n)
    medz[(zc >= 3) & (zc < 8)] = 2
    rhoz[(zc >= 3) & (zc < 8)] = 0.26
    medz[(zc >= 8) & (zc < 10)] = 3
    rhoz[(zc >= 8) & (zc < 10)] = 1.85
    med = np.broadcast_to(medz[:, None, None], (n, n, n)).astype(np.int32).copy()
    rho = np.broadcast_to(rhoz[:, None, None], (n, n, n)).astype(np.float64).copy()
    return Phantom(["H2O521ICRU", "LUNG521ICRU", "ICRPBONE521ICRU"], xb, xb.copy(), zb,
                   med, rho, name="slab64")


CT_MEDIA = ["AIR521ICRU", "LUNG521ICRU", "ICRUTISSUE521ICRU", "ICRPBONE521ICRU"]
CT_THRESHOLDS = (0.1, 0.6, 1.2)  # air < 0.1 <= lung < 0.6 <= tissue < 1.2 <= bone


def ct_phantom(nx=128, ny=128, nz=96, d=0.3, seed=1234, scale=(1.0, 1.0, 1.0)):
    """Seeded CT-like phantom: body ellipsoid (17, 11, 14) cm of soft tissue
    rho~N(1.03, 0.02); two lungs (5, 4, 8) cm centred at x=+-7.5 cm,
    rho~U(0.20, 0.35); a spine cylinder of radius 1.5 cm along z at y=-7 cm,
    rho~U(1.4, 1.9); air (0.0012) outside.  `scale` stretches every shape per
    axis.  Media by density thresholds CT_THRESHOLDS into CT_MEDIA."""
    rng = np.random.default_rng(seed)
    xb = _grid(nx, d, -nx * d / 2)
    yb = _grid(ny, d, -ny * d / 2)
    zb = _grid(nz, d, 0.0)
    sx, sy, sz = scale
    xc = 0.5 * (xb[1:] + xb[:-1])
    yc = 0.5 * (yb[1:] + yb[:-1])
    zc = 0.5 * (zb[1:] + zb[:-1]) - nz * d / 2
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    rho = np.full((nz, ny, nx), 0.0012)
    body = (X / (17 * sx)) ** 2 + (Y / (11 * sy)) ** 2 + (Z / (14 * sz)) ** 2 <= 1.0
    rho[body] = rng.normal(1.03, 0.02, size=int(body.sum()))
    for cx in (-7.5, 7.5):
        lung = ((X - cx * sx) / (5 * sx)) ** 2 + (Y / (4 * sy)) ** 2 + (Z / (8 * sz)) ** 2 <= 1.0
        lung &= body
        rho[lung] = rng.uniform(0.20, 0.35, size=int(lung.sum()))
    spine = (X / (1.5 * sx)) ** 2 + ((Y + 7.0 * sy) / (1.5 * sx)) ** 2 <= 1.0
    spine &= body
    rho[spine] = rng.uniform(1.4, 1.9, size=int(spine.sum()))
    rho = np.round(rho, 6)
    med = np.digitize(rho, CT_THRESHOLDS).astype(np.int32) + 1
    return Phantom(list(CT_MEDIA), xb, yb, zb, med, rho, name=f"ct{nx}x{ny}x{nz}")


def ct_phantom_large(seed=4321):
    """256x256x160 voxels of 0.2 cm, the CT recipe stretched to the extent."""
    return ct_phantom(256, 256, 160, 0.2, seed=seed,
                      scale=(51.2 / 38.4, 51.2 / 38.4, 32.0 / 28.8))


def write_egsphant(path, ph: Phantom):
    """Write the `.egsphant` text format read by omc_dosxyz.c:62-152."""
    nx, ny, nz = ph.shape
    if len(ph.media) > 9:
        raise ValueError("egsphant stores one digit per voxel: at most 9 media")
    lines = [f" {len(ph.media)}"]
    lines += [m for m in ph.media]
    lines.append("  " + " ".join(["0.25"] * len(ph.media)))
    lines.append(f" {nx:5d}{ny:5d}{nz:5d}")
    for b in (ph.xb, ph.yb, ph.zb):
        lines.append(" ".join(f"{v:.6f}" for v in b))
    out = "\n".join(lines) + "\n"
    digits = (ph.med.astype(np.uint8) + ord("0")).astype(np.uint8)
    body = []
    for k in range(nz):
        rows = digits[k].view("S1").reshape(ny, nx)
        body.append("\n".join(r.tobytes().decode() for r in rows) + "\n\n")
    dens = []
    for k in range(nz):
        dens.append("\n".join(" ".join(f"{v:.6f}" for v in row) for row in ph.rho[k]) + "\n\n")
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        f.write(out)
        f.write("".join(body))
        f.write("".join(dens))
    return path


def read_egsphant(path) -> Phantom:
    """Read the `.egsphant` text format (omc_dosxyz.c:62-152)."""
    with open(path) as f:
        nmed = int(f.readline().split()[0])
        media = [f.readline().strip().replace(" ", "") for _ in range(nmed)]
        f.readline()
        nx, ny, nz = (int(v) for v in f.readline().split()[:3])
        vals = []
        while len(vals) < nx + ny + nz + 3:
            vals += [float(v) for v in f.readline().split()]
        xb = np.array(vals[:nx + 1])
        yb = np.array(vals[nx + 1:nx + ny + 2])
        zb = np.array(vals[nx + ny + 2:nx + ny + nz + 3])
        med = np.zeros((nz, ny, nx), dtype=np.int32)
        for k in range(nz):
            for j in range(ny):
                row = f.readline().rstrip("\n")
                med[k, j, :] = np.frombuffer(row[:nx].encode(), dtype=np.uint8) - ord("0")
            f.readline()
        rest = np.array(f.read().split(), dtype=np.float64)
        rho = rest[:nx * ny * nz].reshape(nz, ny, nx)
    return Phantom(media, xb, yb, zb, med, rho, name=Path(path).stem)


# --------------------------------------------------------------------------
# Beam run description and the `.inp` format
# --------------------------------------------------------------------------
@dataclass
class BeamRun:
    """The `.inp` keys omc_dosxyz reads (ucodes/omc_dosxyz/input_file.inp)."""
    phantom_file: str
    spectrum_file: str | None = None
    mono_energy: float = 1.25
    charge: int = 0
    collimator: tuple = (-5.0, 5.0, -5.0, 5.0)
    ssd: float = 100.0
    ncase: int = 100000
    nbatch: int = 10
    seeds: tuple = (97, 33)
    ecut: float = 0.7
    pcut: float = 0.01
    nsplit: int = 1
    pegs_file: str = ""
    pgs4form_file: str = ""
    data_folder: str = ""
    output_folder: str = ""
    extra: dict = field(default_factory=dict)

    def lines(self):
        out = []
        if self.spectrum_file:
            out.append(f"spectrum file = {self.spectrum_file}")
        out.append(f"mono energy = {self.mono_energy}")
        out.append(f"charge = {self.charge}")
        out.append("collimator bounds = " + " ".join(str(v) for v in self.collimator))
        out.append(f"ssd = {self.ssd}")
        out.append(f"ncase = {self.ncase}")
        out.append(f"nbatch = {self.nbatch}")
        out.append(f"rng seeds = {self.seeds[0]} {self.seeds[1]}")
        out.append(f"phantom file = {self.phantom_file}")
        out.append(f"global ecut = {self.ecut}")
        out.append(f"global pcut = {self.pcut}")
        out.append(f"pegs file = {self.pegs_file}")
        out.append(f"pgs4form file = {self.pgs4form_file}")
        out.append(f"nsplit = {self.nsplit}")
        out.append(f"data folder = {self.data_folder}")
        out.append(f"output folder = {self.output_folder}")
        for k, v in self.extra.items():
            out.append(f"{k} = {v}")
        return out


def write_inp(basename, run: BeamRun):
    """Write `<basename>.inp` (ompMC appends `.inp`, omc_utilities.c:68-71)."""
    path = str(basename) + ".inp"
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        f.write("\n".join(run.lines()) + "\n")
    return path


def default_run(phantom_file, spectrum="6mv", root=ASSETS, **kw) -> BeamRun:
    """A BeamRun pointing at the staged physics data."""
    root = Path(root)
    spec = None
    if spectrum:
        spec = str(root / "spectra" / f"{spectrum}.spectrum")
        if not Path(spec).exists():
            write_spectrum(spec, spectrum)
    out = root / "out"
    out.mkdir(parents=True, exist_ok=True)
    base = dict(phantom_file=str(phantom_file), spectrum_file=spec,
                pegs_file=str(root / "pegs4" / "521icru.pegs4dat"),
                pgs4form_file=str(root / "pegs4" / "pgs4form.dat"),
                data_folder=str(root / "data") + "/",
                output_folder=str(out) + "/")
    base.update(kw)
    return BeamRun(**base)


def read_3ddose(path):
    """Read a `.3ddose` file (omc_dosxyz.c:842-879): dims, bounds, dose, unc.
    Returns (dose[nz,ny,nx], unc[nz,ny,nx], (xb, yb, zb))."""
    with open(path) as f:
        nx, ny, nz = (int(v) for v in f.readline().split())
        xb = np.array(f.readline().split(), dtype=np.float64)
        yb = np.array(f.readline().split(), dtype=np.float64)
        zb = np.array(f.readline().split(), dtype=np.float64)
        dose = np.array(f.readline().split(), dtype=np.float64).reshape(nz, ny, nx)
        unc = np.array(f.readline().split(), dtype=np.float64).reshape(nz, ny, nx)
    return dose, unc, (xb, yb, zb)
