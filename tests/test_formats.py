"""Input formats on the host (no GPU): the spectrum inverse CDF the engine
samples from is the reference's bit for bit (initSource,
omc_dosxyz.c:372-503, read back from the reference's own globals), the
.egsphant writer/reader round-trips, and the dosxyz driver rejects each
missing `.inp` key with the reference's message before any device work
(omc_dosxyz.c:69, 525, 597, 609, 823, 904, 910, 1209, 1215)."""
import subprocess
import sys

import numpy as np
import pytest

from tests.conftest import REPO


def reference_cdf(spectrum, tmp_path):
    """initSource's cdfinv1/cdfinv2 for a spectrum, from the reference built
    by oracle/Makefile (run in a child: the reference keeps global state)."""
    from oracle import ref
    ref.build()
    out = tmp_path / f"cdf_{spectrum}.npz"
    code = f"""
import sys; sys.path.insert(0, {str(REPO)!r})
import numpy as np
from ompmc_b200 import assets as A
from oracle.ref import Reference
from tests.golden import make_golden as M
M.WORK.mkdir(parents=True, exist_ok=True)
ph = M.CASES["water30"]["phantom"]()
pf = M.WORK / "water30.egsphant"
if not pf.exists():
    A.write_egsphant(pf, ph)
run = A.default_run(pf, spectrum={spectrum!r}, ncase=1000, nbatch=10)
base = M.WORK / "cdf_{spectrum}"
A.write_inp(base, run)
r = Reference.open(base)
np.savez({str(out)!r}, c1=r.table("cdfinv1"), c2=r.table("cdfinv2"), path=run.spectrum_file)
"""
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-2000:]
    return np.load(out)


@pytest.mark.parametrize("spectrum", ["6mv", "18mv"])
def test_spectrum_cdf_matches_reference(spectrum, tmp_path, assets_root):
    from ompmc_b200.engine import load_spectrum
    ref = reference_cdf(spectrum, tmp_path)
    cdf1, cdf2 = load_spectrum(str(ref["path"]))
    assert len(ref["c1"]) == len(cdf1) > 0
    assert np.array_equal(ref["c1"], cdf1)
    assert np.array_equal(ref["c2"], cdf2)


def test_egsphant_round_trip(tmp_path):
    from ompmc_b200 import assets as A
    ph = A.ct_phantom(20, 16, 12, 0.5, seed=3)
    p = tmp_path / "x.egsphant"
    A.write_egsphant(p, ph)
    q = A.read_egsphant(p)
    assert q.media == ph.media
    for a, b in ((q.xb, ph.xb), (q.yb, ph.yb), (q.zb, ph.zb), (q.rho, ph.rho)):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(q.med, ph.med)


REQUIRED = ["phantom file", "pegs file", "pgs4form file", "data folder", "output folder", "global ecut",
            "global pcut", "nsplit", "collimator bounds", "charge", "ssd", "ncase", "nbatch"]


def _inp_lines(tmp_path):
    from ompmc_b200 import assets as A
    ph = A.water_cube(8, 1.0)
    pf = tmp_path / "w8.egsphant"
    A.write_egsphant(pf, ph)
    run = A.default_run(pf, ncase=1000, nbatch=10, output_folder=str(tmp_path) + "/")
    return run.lines()


@pytest.mark.parametrize("key", REQUIRED)
def test_missing_key_is_rejected_like_the_reference(key, tmp_path, assets_root):
    from ompmc_b200.engine import CLI_PATH
    lines = [l for l in _inp_lines(tmp_path) if not l.split("=")[0].strip().startswith(key)]
    base = tmp_path / "case"
    (tmp_path / "case.inp").write_text("\n".join(lines) + "\n")
    p = subprocess.run([str(CLI_PATH), "-i", str(base), "-o", "out"], capture_output=True, text=True, timeout=120)
    assert p.returncode != 0
    msg = f"Can not find '{key}' key on input file."
    assert msg in p.stdout + p.stderr
    from oracle import ref
    if ref.available():
        r = subprocess.run([str(ref.CLI), "-i", str(base), "-o", "out"], capture_output=True, text=True, timeout=120)
        assert r.returncode != 0
        assert msg in r.stdout + r.stderr


def test_commented_key_counts_as_missing(tmp_path, assets_root):
    """A line with '#' anywhere is skipped (omc_utilities.c:90-96)."""
    from ompmc_b200.engine import CLI_PATH
    lines = [("# " + l if l.startswith("ncase") else l) for l in _inp_lines(tmp_path)]
    (tmp_path / "c.inp").write_text("\n".join(lines) + "\n")
    p = subprocess.run([str(CLI_PATH), "-i", str(tmp_path / "c"), "-o", "out"], capture_output=True, text=True,
                       timeout=120)
    assert p.returncode != 0 and "Can not find 'ncase' key on input file." in p.stdout + p.stderr


def test_sampler_fixtures_reproduce_from_the_oracle(tmp_path):
    """The sampler known answers (tests/golden/kat_slab64.npz) come out of the
    live oracle again, bit for bit, for the first cases of every sampler."""
    import subprocess
    import sys
    from tests.conftest import GOLDEN, REPO
    code = (f"import sys, numpy as np; sys.path.insert(0, {str(REPO)!r}); "
            "from tests.golden import make_golden as M; from oracle.ref import Reference; "
            "M.WORK.mkdir(parents=True, exist_ok=True); "
            "base, ph = M.case_inp('slab64'); r = Reference.open(base); "
            f"g = dict(np.load({str(GOLDEN / 'kat_slab64.npz')!r})); bad = 0; "
            "names = {v: k for k, v in Reference.SAMPLERS.items()}\n"
            "for w in range(10):\n"
            "    key = 'msdist' if w == 9 else names[w]\n"
            "    rn = g[key + '_rn_int'].astype(np.float64) / 16777216.0; off = g[key + '_rn_off']\n"
            "    for c in range(5):\n"
            "        s = rn[off[c]:off[c + 1]]\n"
            "        if w == 9:\n"
            "            us, u, fin = r.msdist(g[key + '_q'][c], *g[key + '_extra'][c], s)\n"
            "            ok = u == g[key + '_used'][c] and us == g[key + '_out'][c, 0, 0] and "
            "np.array_equal(fin, g[key + '_out'][c, 0, 1:7])\n"
            "        else:\n"
            "            u, parts = r.sampler(key, g[key + '_q'][c], s)\n"
            "            ok = u == g[key + '_used'][c] and np.array_equal(parts, g[key + '_out'][c, :len(parts)])\n"
            "        bad += not ok\n"
            "print('BAD', bad)\n")
    from oracle import ref
    ref.build()
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "BAD 0" in p.stdout, p.stdout[-500:]
