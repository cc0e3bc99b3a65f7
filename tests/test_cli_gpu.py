"""The drop-in omc_dosxyz program end to end (omc_dosxyz.c:1072-1307).

ompmc_b200/bin/omc_dosxyz runs on the same `.egsphant`, `.spectrum` and
`.inp` files as the reference CLI (oracle/_ref/omc_dosxyz_ref, built from
the unmodified sources) and writes a `.3ddose` of the same layout: the
header lines (dimensions, voxel boundaries) are byte for byte the
reference's and every number has the reference's printf format.  The dose
of a 2*10^6-history run, in both transport forms, agrees with the
reference's fixture within statistics."""
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import CASES, REPO

pytestmark = pytest.mark.gpu

CLI = REPO / "ompmc_b200" / "bin" / "omc_dosxyz"
REF_CLI = REPO / "oracle" / "_ref" / "omc_dosxyz_ref"


def _inp(tmp_path, ph, name, ncase, nbatch, collimator):
    from ompmc_b200 import assets as A
    pf = tmp_path / f"{name}.egsphant"
    A.write_egsphant(pf, ph)
    run = A.default_run(pf, ncase=ncase, nbatch=nbatch, collimator=collimator, output_folder=str(tmp_path) + "/")
    base = tmp_path / name
    A.write_inp(base, run)
    return base


def _run(exe, base, out, *extra):
    p = subprocess.run([str(exe), "-i", str(base), "-o", out, *extra], capture_output=True, text=True, timeout=600,
                       cwd=str(base.parent))
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return base.parent / f"{out}.3ddose"


def test_3ddose_layout_matches_reference_cli(tmp_path, assets_root):
    if not REF_CLI.exists():
        pytest.skip("reference CLI not built")
    from ompmc_b200 import assets as A
    ph = A.water_cube(8, 1.0)
    base = _inp(tmp_path, ph, "w8", 20000, 10, (-2.0, 2.0, -2.0, 2.0))
    ours = _run(CLI, base, "ours").read_text().splitlines()
    ref = _run(REF_CLI, base, "ref").read_text().splitlines()
    assert len(ours) == len(ref) == 6
    assert ours[:4] == ref[:4]                      # dims and boundaries, byte for byte
    e_fmt = re.compile(r"^-?\d\.\d{6}e[+-]\d{2}$")  # %e
    f_fmt = re.compile(r"^-?\d+\.\d{6}$")           # %f
    for line, fmt in ((4, e_fmt), (5, f_fmt)):
        a, b = ours[line].split(), ref[line].split()
        assert len(a) == len(b) == 8 ** 3
        assert all(fmt.match(t) for t in a) and all(fmt.match(t) for t in b)


@pytest.mark.parametrize("mode", ["event", "plain"])
def test_cli_dose_matches_reference(mode, tmp_path, golden, assets_root):
    from ompmc_b200 import assets as A
    from tests.conftest import case_phantom
    g = golden("dose_water30")
    base = _inp(tmp_path, case_phantom("water30"), "water30", int(g["ncase"]), int(g["nbatch"]),
                CASES["water30"]["collimator"])
    dose, unc, bounds = A.read_3ddose(_run(CLI, base, f"cli_{mode}", "--mode", mode))
    assert dose.shape == tuple(int(v) for v in g["shape"])
    d = dose.ravel()[g["idx"]]
    u = unc.ravel()[g["idx"]]
    sel = g["dose"] > 0.10 * g["dmax"]
    z = (d - g["dose"])[sel] / np.sqrt((u * d) ** 2 + (g["unc"] * g["dose"]) ** 2)[sel]
    assert len(z) > 300
    assert np.mean(np.abs(z) < 3) >= 0.99, np.mean(np.abs(z) < 3)
    assert abs(z.mean()) < 0.25, z.mean()
