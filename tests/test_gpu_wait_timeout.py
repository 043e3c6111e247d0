"""A stalled tensor-core pipeline is reported, not hung.

Every wait inside the tensor-core kernels is bounded (about 2^31 SM clocks, ~1 s); when one
runs out the kernel records a timeout flag, its other roles see the abort and stop, TMEM is
released after the issued MMAs complete, and the call returns DSHT_ERR_CUDA.  The test hook
dsht_test_stall_next_contraction makes the next contraction launch withhold one signal (a
barrier that nothing completes), so that path runs for real; the device stays usable and the
next call is correct."""
import numpy as np
import pytest

from directsht_b200 import DirectSHT
from directsht_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_stalled_contraction_returns_error_and_device_stays_usable():
    rng = np.random.default_rng(0)
    N, Nl, Nx = 20000, 64, 128
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(Nl, Nx, precision="mixed")
    good = d(th, ph, w)
    lib = L.load()
    assert lib.dsht_test_stall_next_contraction() == L.DSHT_OK
    with pytest.raises(L.DSHTError) as e:
        d(th, ph, w)
    assert e.value.code == L.DSHT_ERR_CUDA and "timed out" in e.value.msg
    again = d(th, ph, w)  # the context is intact and the next call is right
    assert np.array_equal(again, good)
