"""GPU tests of the mixed-precision levels, with both bin-sum methods (the NUFFT sums, the
default, and the direct tensor-core sums): results within 1e-7 x max|alm| of the FP64
path, which the parity tests pin to the oracle."""
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
    for bin_sums in ("nufft", "tc", "fp64"):
        d.tune(bin_sums=bin_sums)
        for level in ("mixed", "mixed_f64_tables"):
            d.set_precision(level)
            a = d(th, ph, w)
            assert _rel(a, ref) <= TOL_MIXED, (level, bin_sums)


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

    The tensor-core sums scale their fixed-point operands by the largest |weight| of each
    bin piece, so the error of every point is relative to that largest weight; weight sets
    spanning many more decades lose accuracy on the small weights (see DSHT_PREC_MIXED).
    The NUFFT sums err relative to the bin's sum |w|."""
    rng = np.random.default_rng(9)
    N = 50000
    th = np.arccos(np.concatenate([rng.uniform(0.40, 0.401, N // 2), rng.uniform(-0.7, 0.7, N // 2)]))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.lognormal(0.0, 1.0, N)
    d = DirectSHT(256, 512)
    ref = d.basic_sht(th, ph, w.copy(), verbose=False)
    # Half of the weight sits in one bin: the digit tables' fixed point is relative to each
    # row's and fold column's scale, so both levels hold 1e-7.
    for bin_sums in ("nufft", "tc", "fp64"):
        d.tune(bin_sums=bin_sums)
        for level in ("mixed_f64_tables", "mixed"):
            d.set_precision(level)
            a = d.basic_sht(th, ph, w.copy(), verbose=False)
            assert _rel(a, ref) <= TOL_MIXED, (level, bin_sums)


def _oracle_basic(Nl, Nx, th, ph, w):
    return O.basic_sht(O.build_tables(Nl, Nx), th, ph, w)


@pytest.mark.parametrize("case", ["one_bin", "dominant_bin", "two_bins_signed", "few_points"])
def test_mixed_concentrated_weight_vs_oracle(case):
    """Weight concentrated at a few nodes, against the oracle: the mixed level (tensor-core
    contraction of the 31-bit digit tables) and a compact plan hold 1e-7."""
    rng = np.random.default_rng(11)
    Nl, Nx = 200, 400
    if case == "one_bin":          # every point in one x bin
        N = 30000
        cost = rng.uniform(0.5001, 0.5006, N)
        w = rng.uniform(0.5, 1.5, N)
    elif case == "dominant_bin":    # a fifth of the points in one bin, the rest spread
        N = 40000
        cost = np.concatenate([rng.uniform(-0.1502, -0.15, N // 5), rng.uniform(-0.74, 0.74, N - N // 5)])
        w = rng.lognormal(0.0, 0.5, N)
    elif case == "two_bins_signed":  # two bins on either side of the equator, signed weights
        N = 20000
        cost = np.concatenate([rng.uniform(0.3, 0.3004, N // 2), rng.uniform(-0.6004, -0.6, N // 2)])
        w = rng.normal(1.0, 2.0, N)
    else:                           # fewer points than the tensor-core threshold
        N = 300
        cost = rng.uniform(-0.2, 0.2, N)
        w = rng.uniform(0.5, 1.5, N)
    th = np.arccos(cost)
    ph = rng.uniform(0, 2 * np.pi, N)
    ref = _oracle_basic(Nl, Nx, th, ph, w)
    for kwargs in (dict(precision="mixed"), dict(compact_tables=True)):
        d = DirectSHT(Nl, Nx, **kwargs)
        for bin_sums in ("nufft", "tc", "fp64"):
            d.tune(bin_sums=bin_sums)
            a = d.basic_sht(th, ph, w.copy(), verbose=False)
            assert _rel(a, ref) <= TOL_MIXED, (case, kwargs, bin_sums)


@pytest.mark.parametrize("N,seed", [(1, 0), (700, 1), (5000, 2)])
def test_compact_plan_few_points_call_vs_oracle(N, seed):
    """A compact-table plan (no FP64 tables at all) on a handful of points, polar ones
    included (FP64 bin sums, tensor-core contraction of the digit tables)."""
    rng = np.random.default_rng(seed)
    Nl, Nx = 96, 192
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    ref = O.direct_sht(O.build_tables(Nl, Nx), th, ph, w)
    d = DirectSHT(Nl, Nx, compact_tables=True)
    assert _rel(d(th, ph, w), ref) <= TOL_MIXED


@pytest.mark.slow
def test_compact_plan_nl2048_concentrated_columns_vs_oracle():
    """Nl=2048, Nx=4096 with compact tables only (68.7 GB, the uneven-batch and serving plans at
    that size): 40 % of the weight in one bin, the rest spread; columns against the per-m
    oracle."""
    rng = np.random.default_rng(12)
    Nl, Nx, N = 2048, 4096, 400_000
    cost = np.concatenate([rng.uniform(0.2000, 0.2001, 2 * N // 5), rng.uniform(-0.74, 0.74, N - 2 * N // 5)])
    th = np.arccos(cost)
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(Nl, Nx, compact_tables=True)
    a = d.basic_sht(th, ph, w.copy(), verbose=False)
    cols = {m: O.basic_sht_column(Nl, Nx, 0.75, m, th, ph, w) for m in (0, 1, 2, 700, 1500, 2047)}
    scale = max(np.abs(c).max() for c in cols.values())
    for m, col in cols.items():
        r0 = O.healpy_index(m, m, Nl)
        assert np.abs(a[r0:r0 + Nl - m] - col).max() <= TOL_MIXED * scale, m


@pytest.mark.slow
def test_mixed_c2_full_size():
    """Survey-like single map, Nl=1024, Nx=2048, N=1e7: mixed within 1e-7 of FP64."""
    rng = np.random.default_rng(0)
    N = 10_000_000
    th = np.arccos(rng.uniform(np.cos(1.2), np.cos(0.3), N))
    ph = rng.uniform(0, 1.5 * np.pi, N)
    w = rng.lognormal(0.0, 0.5, N)
    d = DirectSHT(1024, 2048)
    ref = d(th, ph, w)
    d.set_precision("mixed")
    for bin_sums in ("nufft", "tc", "fp64"):
        d.tune(bin_sums=bin_sums)
        a = d(th, ph, w)
        assert _rel(a, ref) <= TOL_MIXED, bin_sums
