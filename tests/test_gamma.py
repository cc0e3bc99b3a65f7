"""Gamma index (ompmc_b200.gamma) on analytic distributions: identical
doses pass with gamma 0, a 3 % global scaling fails in the flat high-dose
region and passes where it is below 2 % of the maximum, a 1 mm shift of a
steep gradient passes 2 %/2 mm although the dose difference alone fails,
and a 3 mm shift fails there."""
import numpy as np

from ompmc_b200.gamma import gamma_index, gamma_pass_rate


def grid(n=40, d=0.1):
    b = np.arange(n + 1) * d
    return b, b.copy(), b.copy()


def field(shift=0.0, n=40, d=0.1):
    """Penumbra along x (error function, 3 mm wide), flat in y and z."""
    from math import erf
    xb, yb, zb = grid(n, d)
    cx = 0.5 * (xb[:-1] + xb[1:])
    prof = np.array([0.5 * (1 - erf((x - 2.0 - shift) / 0.15)) for x in cx])
    return np.broadcast_to(prof[None, None, :], (n, n, n)).copy(), (xb, yb, zb)


def test_identical_passes_with_zero_gamma():
    d, b = field()
    idx = np.arange(d.size)
    rate, g = gamma_pass_rate(idx, d.ravel(), d, b)
    assert rate == 1.0 and np.allclose(g, 0.0)


def test_global_scaling():
    d, b = field()
    idx = np.arange(d.size)
    g = gamma_index(idx, d.ravel(), 1.03 * d, b, dd=0.02, dta=0.2)
    ref = d.ravel()
    flat_high = ref > 0.99999                   # more than 2 mm from the penumbra
    assert flat_high.sum() > 1000
    assert np.all(g[flat_high] > 1.0)          # 3 % of Dmax where the dose is flat
    low = ref < 0.5
    assert np.all(g[low] <= 1.0)               # 3 % of < 50 % Dmax is < 2 % of Dmax


def test_shift_inside_dta_passes_outside_fails():
    d, b = field()
    d1, _ = field(shift=0.1)                    # 1 mm
    d3, _ = field(shift=0.3)                    # 3 mm
    idx = np.arange(d.size)
    ref = d.ravel()
    grad = (ref > 0.2) & (ref < 0.8)
    dd_only = np.abs(d1.ravel() - ref)[grad] > 0.02
    assert dd_only.mean() > 0.5                 # the dose difference alone fails there
    g1 = gamma_index(idx[grad], ref[grad], d1, b, dd=0.02, dta=0.2, d_norm=1.0)
    assert np.all(g1 <= 1.0)
    g3 = gamma_index(idx[grad], ref[grad], d3, b, dd=0.02, dta=0.2, d_norm=1.0)
    assert np.mean(g3 > 1.0) > 0.9
