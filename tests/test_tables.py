"""Host table builder vs the reference's in-memory tables, element by element
(ompMC initMediaData, src/ompmc.c:5468; the reference is built from its own
sources by oracle/Makefile and dumped through oracle/harness.c).

Bit-exact everywhere except two documented spots where the reference reads
memory it never wrote: the last Rayleigh power-law exponent (b_array[99],
c_array[99], never read by the sampler) and the positron screening table
etap_ms above beta^2 = b2spin_max, where the reference interpolates with one
element past its eta array (ompmc.c:2690-2745); this engine clamps there."""
import subprocess
import sys

import numpy as np
import pytest

from tests.conftest import CASES, REPO

pytestmark = pytest.mark.filterwarnings("ignore::RuntimeWarning")


def reference_tables(case, tmp_path, spin=False):
    from oracle import ref
    ref.build()
    out = tmp_path / f"ref_{case}.npz"
    what = "_tablesspin" if spin else "_tables"
    code = (f"import sys; sys.path.insert(0, {str(REPO)!r}); "
            f"from tests.golden import make_golden as M; M.WORK.mkdir(parents=True, exist_ok=True); "
            f"M.{what}({case!r}, {str(out)!r})")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-2000:]
    return dict(np.load(out))


def etap_exact_bins(tables, nmed):
    """Bins whose upper energy is below the last beta^2 node of the spin grid."""
    e_arr = tables.get("e_array").reshape(nmed, 500)
    s = tables.get("spin_scalars")
    b2min, dbeta2i = s[0], s[1]
    b2max = b2min + 15.0 / dbeta2i
    tau = e_arr / 0.5109989461
    beta2 = tau * (tau + 2) / (tau + 1) ** 2
    ok = np.zeros_like(e_arr, dtype=bool)
    ok[:, :-1] = beta2[:, 1:] < b2max - 1e-9
    # the last bin of each medium repeats the previous one; the grid beyond
    # meke is zero-filled
    meke = tables.get("meke")
    for m in range(nmed):
        ok[m, meke[m]:] = False
        ok[m, :meke[m]] = np.logical_and.accumulate(ok[m, :meke[m] - 1].tolist() + [ok[m, meke[m] - 2]])
    return ok


@pytest.mark.parametrize("case,spin", [(c, False) for c in CASES] + [("slab64", True), ("ctsmall", True)])
def test_tables_match_reference(case, spin, tmp_path, assets_root):
    """spin: the data folder with the synthetic, non-constant spin file, whose
    rejection surface and moment corrections differ from 1."""
    from ompmc_b200 import assets as A
    from ompmc_b200.engine import Tables
    if spin:
        A.stage_spin_variant(assets_root)
    ref = reference_tables(case, tmp_path, spin)
    media = CASES[case]["media"]
    nmed = len(media)
    t = Tables.from_assets(media, assets_root, data="data_spin" if spin else "data")
    if spin:
        # the variant really differs from the neutral file
        sr = t.get("spin_rej")
        assert sr.min() < 0.5 and sr.max() == 1.0
        q1 = t.get("q1ce_ms0")
        assert np.any(np.abs(q1[q1 != 0] - 1.0) > 0.01)
    ok_etap = etap_exact_bins(t, nmed)
    bad = []
    for name, a in ref.items():
        if name.startswith("s_"):
            continue
        b = t.get(name)
        assert a.shape == b.shape, name
        if name in ("b_array", "c_array"):
            a, b = a.reshape(nmed, 100)[:, :99], b.reshape(nmed, 100)[:, :99]
        elif name in ("wms", "ims"):
            a, b = a.reshape(-1, 32)[:, :31], b.reshape(-1, 32)[:, :31]
        elif name in ("etap_ms0", "etap_ms1"):
            a, b = a.reshape(nmed, 500)[ok_etap], b.reshape(nmed, 500)[ok_etap]
        if not np.array_equal(a, b):
            rel = np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-300))
            bad.append((name, rel))
    assert not bad, f"tables differ from the reference: {bad}"
    s = t.get("spin_scalars")
    for i, k in enumerate(["b2spin_min", "dbeta2i", "espml", "dleneri", "dqq1i", "dllambi", "dqmsi"]):
        assert s[i] == ref["s_" + k], k


def test_etap_deviation_is_confined_to_top_bins(assets_root):
    from ompmc_b200.engine import Tables
    t = Tables.from_assets(["H2O521ICRU"], assets_root)
    ok = etap_exact_bins(t, 1)
    meke = int(t.get("meke")[0])
    # only bins above ~15.6 MeV are excluded from the exact comparison
    e_arr = t.get("e_array")[:meke]
    assert e_arr[np.argmin(ok[0, :meke])] > 15.0
    assert ok[0, :meke].sum() >= meke - 30
