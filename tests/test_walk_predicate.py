"""The walk's neighbour test for lists built with a skin (csrc/kernels_walk.cu, near_sources).

Lists built with a skin are candidate sets: the gather kernels keep a pair only when r < h_ij at the current
smoothing lengths, and the smoothing-length solve holds each h below h0·(1 + skin)·0.999. The walk therefore
uses a conservative one-FMA test, d² < lim'² with lim' = fma(h_j, c, h_i·c), c = ½(1 + skin)(1 + 2⁻¹⁹), in
place of the exact predicate sqrt_rn(d²) < ½(h_i + h_j)(1 + skin) that it used before. The float32 arithmetic
of both is restated here and sampled at the support boundary:

1. every pair the exact predicate admits, the conservative test admits (the new list contains the old one);
2. every pair a gather pass can still accept, once h has grown to its cap and with the approximate reciprocal
   square root's error, is in the list.

With both, the sums of every gather pass see the same neighbours in the same order as with the exact list.
"""
import numpy as np
import pytest

f32 = np.float32
PAD = f32(1.0) + f32(1.9073486e-6)  # 1 + 2^-19


def _fma32(a, b, c):
    """fmaf: the product of two float32 values is exact in float64; one rounding of the sum (to float32) after
    one in float64 can differ from a single rounding by at most one float32 ulp, far inside the 2^-19 pad."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(f32)


def _exact_inside(dd, hi, hj, skin):
    lim = (f32(0.5) * (hi + hj)).astype(f32) * (f32(1.0) + skin)
    return np.sqrt(dd) < lim  # float32 sqrt is correctly rounded in numpy


def _loose_inside(dd, hi, hj, skin):
    lim_j = (f32(0.5) * (f32(1.0) + skin)) * PAD
    lim_i = hi * lim_j
    lim = _fma32(hj, np.full_like(hj, lim_j), lim_i)
    return dd < lim * lim


def _boundary_pairs(rng, n, skin, spread):
    hi = (10.0 ** rng.uniform(-3, 6, n)).astype(f32)
    hj = (hi * rng.uniform(0.7, 1.3, n)).astype(f32)
    lim = 0.5 * (hi.astype(np.float64) + hj.astype(np.float64)) * (1.0 + float(skin))
    dd = ((lim * (1.0 + rng.uniform(-spread, spread, n))) ** 2).astype(f32)
    return dd, hi, hj


@pytest.mark.parametrize("skin", [f32(1.0e-5), f32(0.05), f32(0.15), f32(0.5)])
def test_conservative_test_contains_the_exact_predicate(skin):
    rng = np.random.default_rng(int(skin * 1e6) + 1)
    for spread in (1e-3, 1e-6):
        dd, hi, hj = _boundary_pairs(rng, 400_000, skin, spread)
        exact = _exact_inside(dd, hi, hj, skin)
        loose = _loose_inside(dd, hi, hj, skin)
        assert exact.any() and (~exact).any()
        assert not (exact & ~loose).any()
        if spread == 1e-3:
            # a tight superset: the extra pairs lie in the pad's band, |r/lim − 1| ≲ 2^-19 of the ±1e-3 sampled
            # (about (2^-19 / 1e-3) / 2 of the pairs), plus the rounding of either form
            assert (loose & ~exact).sum() <= 2.0 * 2.0 ** -19 / spread * len(dd)


@pytest.mark.parametrize("skin", [f32(0.05), f32(0.15), f32(0.5)])
def test_every_pair_a_gather_pass_can_accept_is_listed(skin):
    """The gather kernels compute r = d²·rsqrt(d²) (approximate, relative error below 2^-22) and
    h_ij = ½(h_i' + h_j') with h' at most h0·(1 + skin)·0.999."""
    rng = np.random.default_rng(7)
    dd, hi, hj = _boundary_pairs(rng, 400_000, skin, 5e-3)
    cap = (f32(1.0) + skin) * f32(0.999)
    hi2, hj2 = (hi * cap).astype(f32), (hj * cap).astype(f32)
    r_low = (np.sqrt(dd.astype(np.float64)) * (1.0 - 2.0 ** -22)).astype(f32)  # the smallest r it can compute
    gather_accepts = r_low < (f32(0.5) * (hi2 + hj2)).astype(f32)
    assert gather_accepts.any()
    assert not (gather_accepts & ~_loose_inside(dd, hi, hj, skin)).any()
