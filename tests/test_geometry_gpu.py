"""Geometry walk parity: the FP64 device howfar/hownear against the reference
ucode (omc_dosxyz.c:187-334) on identical rays — every call's distance,
new region and discard flag must be bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["water30", "slab64", "ctsmall"])
def test_walk_bit_exact(case, golden, engine_for):
    g = golden(f"rays_{case}")
    eng = engine_for(case)
    cap = int(g["cap"])
    us, irn, idc, nc, hn = eng.trace_rays(g["rays"], cap=cap)
    assert np.array_equal(nc, g["ncalls"])
    for r in range(len(nc)):
        n = nc[r]
        assert np.array_equal(us[r, :n], g["ustep"][r, :n]), f"ray {r}: ustep differs"
        assert np.array_equal(irn[r, :n], g["irnew"][r, :n]), f"ray {r}: irnew differs"
        assert np.array_equal(idc[r, :n], g["idisc"][r, :n]), f"ray {r}: idisc differs"
    assert np.array_equal(hn, g["hownear"])
    # every ray ends by leaving the phantom (discard on region 0)
    assert all(idc[r, nc[r] - 1] == 1 for r in range(len(nc)))
