"""Trajectory parity: FP64 device transport replayed on the uniform streams the
reference consumed, history by history.

The reference (single thread, RANMAR) recorded for each history its primary,
every random number it drew and every deposit (region, weighted energy)
(tests/golden/make_golden.py).  The device physics draws random numbers in the
reference's order, so on the same stream it must consume exactly the same
count and reproduce the deposit sequence.  The bar is what the device
achieves on every fixture: all histories match exactly in random-number
count and deposit regions, with energies within 1e-9 relative, and the
total deposit of all histories agrees within 1e-12 relative (measured:
every history exact, totals within 6e-16).  The mismatch count and the
aggregate difference are printed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def replay_case(case, golden, engine_for, fixture="replay"):
    g = golden(f"{fixture}_{case}")
    rn = g["rn_int"].astype(np.float64) / 16777216.0
    ns = int(g.get("nsplit", 1))
    data = "data_spin" if fixture == "replayspin" else "data"
    eng = engine_for(case, data=data, nsplit=ns) if ns > 1 else engine_for(case, data=data)
    dir_, de, nd, nu, fl = eng.replay(g["prim"], rn, g["rn_off"], dep_cap=8192)
    return g, dir_, de, nd, nu, fl


@pytest.mark.parametrize("case", ["water30", "slab64", "ctsmall"])
@pytest.mark.parametrize("fixture", ["replay", "replaysplit", "replayspin"])
def test_replay_matches_reference(fixture, case, golden, engine_for):
    """replaysplit: photon splitting with nsplit = 20 (each photon
    interaction sampled 20 times at weight 1/20, Russian roulette of photons
    made by electrons), the sample input's setting.  replayspin: the
    synthetic spin file, so the Mott/spin rejection of the multiple
    scattering sampler and the moment corrections of the MS step act (with
    the neutral file the rejection surface is 1 everywhere)."""
    g, dir_, de, nd, nu, fl = replay_case(case, golden, engine_for, fixture)
    nh = len(g["prim"])
    rn_len = np.diff(g["rn_off"])
    d_len = np.diff(g["d_off"])
    exact = 0
    mismatched = []
    for h in range(nh):
        ref_ir = g["dep_ir"][g["d_off"][h]:g["d_off"][h + 1]]
        ref_e = g["dep_e"][g["d_off"][h]:g["d_off"][h + 1]]
        ok = (nu[h] == rn_len[h] and nd[h] == d_len[h] and fl[h] == 0
              and np.array_equal(dir_[h, :nd[h]], ref_ir)
              and np.allclose(de[h, :nd[h]], ref_e, rtol=1e-9, atol=1e-12))
        exact += ok
        if not ok:
            mismatched.append(h)
    tot_ref = g["dep_e"].sum()
    tot = sum(de[h, :nd[h]].sum() for h in range(nh))
    print(f"replay {fixture}_{case}: {nh - exact}/{nh} histories differ {mismatched[:10]}; "
          f"aggregate deposit rel. diff {abs(tot - tot_ref) / abs(tot_ref):.3e}")
    assert exact == nh, f"{case}: only {exact}/{nh} histories match; first mismatches {mismatched[:10]}"
    assert abs(tot - tot_ref) <= 1e-12 * abs(tot_ref)


def test_replay_flags_exhausted_stream(golden, engine_for):
    """A truncated stream is reported by a flag, not a fault or a hang."""
    g = golden("replay_water30")
    rn = g["rn_int"].astype(np.float64) / 16777216.0
    off = g["rn_off"]
    hs = [h for h in range(len(off) - 1) if off[h + 1] - off[h] > 40][:3]
    # each history gets the first 5 numbers of its own recorded stream
    rn5 = np.concatenate([rn[off[h]:off[h] + 5] for h in hs])
    short = np.arange(len(hs) + 1, dtype=np.int64) * 5
    eng = engine_for("water30")
    _, _, _, nu, fl = eng.replay(g["prim"][hs], rn5, short, dep_cap=4096)
    assert all(fl & 8), fl
    assert all(nu > 5)
