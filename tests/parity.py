"""Shared parity checks of the GPU tests."""
import numpy as np


def assert_final_rounding(got32, e64):
    """got32 is e64 rounded to float: within half an ulp (the device's bg may
    differ from the host's long double evaluation in the last double bits,
    far below a float ulp)."""
    got = got32.astype(np.float64)
    half_ulp = 0.5 * np.spacing(np.abs(got32)).astype(np.float64)
    dev = np.abs(got - e64)
    assert np.all(dev <= half_ulp * (1 + 1e-6) + 1e-15 * np.abs(e64)), (dev / half_ulp).max()
    assert np.mean(got32 == e64.astype(np.float32)) > 0.999
