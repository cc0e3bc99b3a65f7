"""Known-answer tests of every interaction sampler and of msdist, against the
unmodified reference on the same scripted streams.

tests/golden/kat_<case>.npz holds, per sampler (compton, photo, pair,
rayleigh, moller, bhabha, brems, annih, rannih) and for msdist, 120 seeded
particles in random voxels of the phantom, the uniform stream each case may
draw from, and what the reference returned: its particle stack after the
call (msdist: the step length and final position and direction) and the
count of random numbers it drew (tests/golden/make_golden.py, `_kat`).
The device runs the FP64 sampler of the plain form on each case
(omc_kat).  Exact agreement is expected: the same draws in the same order
and the same arithmetic, up to last-bit differences of libm and CUDA's
transcendental functions.  The bar is what the device achieves: in every
case every sampler draws the same count of numbers and returns the same
particles (as a set; 1e-10 relative); mismatches are printed.  msdist cases of positrons above 15 MeV are left
out: there the reference reads its positron screening table past the end
(see POSITRON_ETA_LIMIT_MEV).  katspin_: the synthetic spin file, which the
multiple-scattering sampler inside msdist reads (spin rejection, moment
corrections)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SAMPLERS = ["compton", "photo", "pair", "rayleigh", "moller", "bhabha", "brems", "annih", "rannih"]


def _sorted_parts(o, n):
    """The first n particles (10 fields each) ordered by charge then energy."""
    p = o[:n, :10]
    return p[np.lexsort((p[:, 6], p[:, 9]))]


# Positrons whose msdist step energy lies in the electron-grid bins above
# beta^2 = b2spin_max (15.6 MeV with the stand-in spin files): there the
# reference interpolates its positron screening table with one element past
# its eta array (ompmc.c:2690-2745, heap memory it never wrote), which this
# engine clamps; such cases have no defined reference answer.
POSITRON_ETA_LIMIT_MEV = 15.0


def _defined(key, q):
    if key != "msdist":
        return np.ones(len(q), dtype=bool)
    return ~((q[:, 9] > 0) & (q[:, 6] - 0.5109989461 > POSITRON_ETA_LIMIT_MEV))


def _compare(g, eng, key):
    q = g[f"{key}_q"]
    rn = g[f"{key}_rn_int"].astype(np.float64) / 16777216.0
    off = g[f"{key}_rn_off"]
    extra = g.get(f"{key}_extra")
    out, nout, used, flags = eng.kat(key, q, rn, off, extra)
    ref_out, ref_n, ref_used = g[f"{key}_out"], g[f"{key}_nout"], g[f"{key}_used"]
    bad = []
    defined = _defined(key, q)
    for c in range(len(q)):
        if not defined[c]:
            continue
        ok = used[c] == ref_used[c] and flags[c] == 0 and nout[c] == ref_n[c]
        if ok and key == "msdist":
            ok = np.allclose(out[c, 0, :7], ref_out[c, 0, :7], rtol=1e-10, atol=1e-13)
        elif ok:
            ok = np.allclose(_sorted_parts(out[c], nout[c]), _sorted_parts(ref_out[c], ref_n[c]), rtol=1e-10,
                             atol=1e-13)
        if not ok:
            bad.append(c)
    return bad, int(defined.sum())


@pytest.mark.parametrize("case", ["slab64", "ctsmall"])
@pytest.mark.parametrize("key", SAMPLERS + ["msdist"])
def test_sampler_matches_reference(case, key, golden, engine_for):
    g = golden(f"kat_{case}")
    bad, n = _compare(g, engine_for(case), key)
    print(f"kat {case} {key}: {len(bad)}/{n} cases differ {bad[:10]}")
    assert not bad, f"{key} on {case}: {len(bad)}/{n} cases differ from the reference: {bad[:10]}"


def test_msdist_with_spin_matches_reference(golden, engine_for):
    g = golden("katspin_slab64")
    bad, n = _compare(g, engine_for("slab64", data="data_spin"), "msdist")
    print(f"katspin slab64 msdist: {len(bad)}/{n} cases differ {bad[:10]}")
    assert not bad, f"msdist with spin: {len(bad)}/{n} cases differ: {bad[:10]}"
