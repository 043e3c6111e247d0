"""GPU tests of the mixed-precision path (tensor-core per-bin sums): results within
1e-7 x max|alm| of the FP64 path, which the parity tests pin to the oracle."""
import numpy as np
import pytest

import inputs as I
from directsht_b200 import DirectSHT
from oracle import dsht_oracle as O

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-7


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _golden(name):
    return np.load(f"{I.__file__.rsplit('/', 1)[0]}/{name}.npz")


@pytest.mark.parametrize("name", ["c1_full_sky", "small_call", "cap_c2like", "small_basic_mixed_sign",
                                  "one_bin", "nodes_exact", "test_alm_example", "single_point"])
def test_mixed_matches_reference_golden(name):
    s = I.CASES[name]
    g = _golden(name)
    th, ph, w = I.make_inputs(name)
    d = DirectSHT(s["Nl"], s["Nx"], s.get("xmax", 0.75), precision="mixed")
    if s["entry"] == "call":
        a = d(th, ph, w)
    else:
        a = d.basic_sht(th, ph, w.copy(), reg_factor=s.get("reg", 1.0), verbose=False)
    assert _rel(a, g["alm"]) <= TOL_MIXED


@pytest.mark.parametrize("Nl,Nx,N,seed", [(1, 2, 10, 0), (9, 20, 300, 1), (100, 200, 5000, 2),
                                          (129, 256, 20000, 3), (300, 600, 50000, 4), (600, 1200, 100000, 5),
                                          (1024, 2048, 200000, 6), (1500, 3000, 100000, 7),
                                          (2048, 4096, 50000, 8)])
def test_mixed_matches_fp64(Nl, Nx, N, seed):
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.lognormal(0, 0.5, N)
    d = DirectSHT(Nl, Nx)
    ref = d(th, ph, w)
    for level in ("mixed", "mixed_f64_tables"):
        d.set_precision(level)
        a = d(th, ph, w)
        assert _rel(a, ref) <= TOL_MIXED, level


def test_small_transforms_use_fp64_sums():
    """Below the threshold the mixed plan runs the FP64 sums: identical to the FP64 plan."""
    from directsht_b200 import _lib as L
    nmin = L.load().dsht_mixed_min_points()
    assert nmin == 1024
    rng = np.random.default_rng(10)
    N = nmin - 1
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(64, 128)
    ref = d(th, ph, w)
    d.set_precision("mixed")
    assert np.array_equal(d(th, ph, w), ref) or _rel(d(th, ph, w), ref) <= 1e-15


def test_mixed_heavy_bin_and_wide_weights():
    """Many points in one bin (several pieces) and lognormal(0, 1) weights.

    The fixed-point operands are scaled by the largest |weight| of each bin piece, so the
    error of every point is relative to that largest weight; weight sets spanning many
    more decades lose accuracy on the small weights (see DSHT_PREC_MIXED)."""
    rng = np.random.default_rng(9)
    N = 50000
    th = np.arccos(np.concatenate([rng.uniform(0.40, 0.401, N // 2), rng.uniform(-0.7, 0.7, N // 2)]))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.lognormal(0.0, 1.0, N)
    d = DirectSHT(256, 512)
    ref = d.basic_sht(th, ph, w.copy(), verbose=False)
    # Half of the weight sits in one bin: the FP32 table rounding does not average out, so
    # the level with FP64 tables is the one held to 1e-7; the FP32-table level stays within
    # a few 1e-7.
    d.set_precision("mixed_f64_tables")
    a = d.basic_sht(th, ph, w.copy(), verbose=False)
    assert _rel(a, ref) <= TOL_MIXED
    d.set_precision("mixed")
    a = d.basic_sht(th, ph, w.copy(), verbose=False)
    assert _rel(a, ref) <= 5 * TOL_MIXED


@pytest.mark.slow
def test_mixed_c2_full_size():
    """Nl=1024, Nx=2048, N=1e7 -- mixed within 1e-7 of FP64."""
    rng = np.random.default_rng(0)
    N = 10_000_000
    th = np.arccos(rng.uniform(np.cos(1.2), np.cos(0.3), N))
    ph = rng.uniform(0, 1.5 * np.pi, N)
    w = rng.lognormal(0.0, 0.5, N)
    d = DirectSHT(1024, 2048)
    ref = d(th, ph, w)
    d.set_precision("mixed")
    a = d(th, ph, w)
    assert _rel(a, ref) <= TOL_MIXED
