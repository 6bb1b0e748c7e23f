"""The Check2 selector thresholds of the BC1 trial error loop (quicktex_b200/csrc/qt_bc1_thread.cuh,
check2_threshold), checked exhaustively on the CPU in IEEE float32.

FindSelectors' Check2 mode (BC1Encoder.cpp:723-729) projects each texel onto the palette axis and
takes sl = clamp(trunc(fl(fl(dd * f) + 0.5)), 1, 3), with dd = (p - c0).axis an exact integer and
f = fl(4 / fl(|axis|^2 + 0.00000125)). The encoder instead compares dd with two integer
thresholds per trial: the smallest dd with fl(fl(dd * f) + 0.5) >= s, for s = 2 and 3. It finds
each as est + (rounded expression at est < s), est = ceil(fl(fl(s - 0.5) * fl(den / 4))). This
test proves, for every |axis|^2 the encoder can meet (0 .. 3 * 255^2), that the rounded
expression is monotone in dd around the threshold and that the threshold is est or est + 1.
"""

import numpy as np

f32 = np.float32


def _pred(dd, f, s):
    return (dd.astype(f32) * f + f32(0.5)) >= f32(s)


def test_thresholds_exhaustive():
    n2 = np.arange(0, 3 * 255 * 255 + 1, dtype=np.int64)
    den = n2.astype(f32) + f32(0.00000125)
    f = f32(4.0) / den
    assert f.dtype == np.float32
    quarter = den * f32(0.25)
    for s in (2, 3):
        est = np.ceil((f32(s) - f32(0.5)) * quarter).astype(np.int64)
        # the encoder's threshold
        t_enc = est + (~_pred(est, f, s)).astype(np.int64)
        # the true threshold, by scanning a window around the estimate
        lo = est - 8
        prev = _pred(lo - 1, f, s)
        assert not prev.any()
        true_t = np.full(n2.shape, -1, dtype=np.int64)
        for k in range(17):
            p = _pred(lo + k, f, s)
            assert (p >= prev).all()  # monotone
            newly = p & (true_t < 0) & ~prev
            true_t[newly] = (lo + k)[newly]
            prev = p
        assert (true_t >= lo).all()
        np.testing.assert_array_equal(t_enc, true_t)


def test_thresholds_match_selector_formula():
    """Spot check on sampled (axis, dd) pairs: dd >= threshold(s) exactly when the clamped selector >= s."""
    rng = np.random.default_rng(7)
    n2 = rng.integers(0, 3 * 255 * 255 + 1, 20000)
    dd = rng.integers(-3 * 255 * 255, 3 * 255 * 255 + 1, 20000)
    den = n2.astype(f32) + f32(0.00000125)
    f = f32(4.0) / den
    sl = np.clip(np.trunc(dd.astype(f32) * f + f32(0.5)), 1, 3).astype(np.int64)
    for s in (2, 3):
        est = np.ceil((f32(s) - f32(0.5)) * (den * f32(0.25))).astype(np.int64)
        t = est + (~_pred(est, f, s)).astype(np.int64)
        np.testing.assert_array_equal(dd >= t, sl >= s)
