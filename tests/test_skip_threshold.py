"""The posterior skips of the exact statistics (vl/fisher.c:440: q < 1e-6;
vl/gmm.c:1099: q < 1e-2/K) compare a float posterior with a double threshold.
The sparse statistics kernel compares the float itself with tf, the smallest
float at or above the threshold, formed on the host as (float)t, raised by one
ulp when that rounded below t.  These tests check, for every float within 64
ulps of tf and for the thresholds the library uses, that the two compares agree
(NaN passes both: neither compare is true for it)."""
import numpy as np
import pytest


def smallest_float_at_or_above(t: float) -> np.float32:
    tf = np.float32(t)
    if float(tf) < t:
        tf = np.nextafter(tf, np.float32(np.inf))
    return tf


def neighbourhood(tf: np.float32, n: int = 64) -> np.ndarray:
    bits = np.int64(np.array([tf], np.float32).view(np.int32)[0])
    return (bits + np.arange(-n, n + 1)).astype(np.int32).view(np.float32)


THRESHOLDS = [1e-6] + [1e-2 / k for k in range(1, 4097)]


@pytest.mark.parametrize("chunk", range(0, len(THRESHOLDS), 512))
def test_float_compare_matches_double_compare(chunk):
    for t in THRESHOLDS[chunk:chunk + 512]:
        tf = smallest_float_at_or_above(t)
        assert float(tf) >= t and float(np.nextafter(tf, np.float32(0))) < t
        v = neighbourhood(tf)
        assert np.array_equal(v.astype(np.float64) < t, v < tf), t


def test_nan_and_signed_zero():
    tf = smallest_float_at_or_above(1e-6)
    for v in (np.float32(np.nan), np.float32(-0.0), np.float32(0.0), np.float32(-np.inf)):
        assert bool(np.float64(v) < 1e-6) == bool(v < tf)
