"""The tensor-core contraction (contract_tc.cu) of the 4-byte digit tables (digits.cu).

With fewer than 1024 points the bin sums are FP64, so the difference to the FP64 plan is the
contraction's own (fixed-point tables and folds, integer digit classes): held to 1e-9 x
max|alm| here, far inside the mixed level's 1e-7.  Larger sets run the tensor-core bin sums
too and are held to 1e-7.  Several maps or point sets share one contraction pass."""
import numpy as np
import pytest
import torch

from directsht_b200 import DirectSHT
from oracle import dsht_oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _full_sky(N, seed, wkind="uniform"):
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N) if wkind == "uniform" else rng.normal(0.0, 1.0, N)
    return th, ph, w


@pytest.mark.parametrize("Nl,Nx,N", [(1, 2, 500), (2, 3, 900), (16, 32, 1000), (64, 130, 1000), (129, 250, 700),
                                     (300, 600, 1000)])
def test_digit_contraction_alone_vs_oracle(Nl, Nx, N):
    th, ph, w = _full_sky(N, Nl)
    ref = O.direct_sht(O.build_tables(Nl, Nx), th, ph, w)
    for kw in (dict(precision="mixed"), dict(compact_tables=True)):
        d = DirectSHT(Nl, Nx, **kw)
        assert _rel(d(th, ph, w), ref) <= 1e-9, kw


@pytest.mark.parametrize("Nl,Nx,N", [(64, 128, 30000), (200, 400, 100000), (513, 1030, 200000)])
def test_mixed_level_vs_fp64(Nl, Nx, N):
    th, ph, w = _full_sky(N, 7 + Nl)
    d = DirectSHT(Nl, Nx)
    ref = d(th, ph, w)
    d.set_precision("mixed")
    a = d(th, ph, w)
    assert _rel(a, ref) <= 1e-7
    assert np.array_equal(a, d(th, ph, w))  # deterministic


def test_signed_zero_mean_weights():
    """Weights of both signs summing to about zero, so that max|alm| is far below sum|w| and
    the fold columns' scales (bounds from sum |w| per node) are loose.  The contraction
    alone (FP64 bin sums below 1024 points) stays within 1e-9 of the oracle, and with the
    NUFFT bin sums it differs from the FP64-table contraction of the same bin sums by less
    than 1e-8."""
    Nl, Nx = 128, 256
    th, ph, w = _full_sky(900, 3, wkind="normal")
    ref = O.direct_sht(O.build_tables(Nl, Nx), th, ph, w)
    d = DirectSHT(Nl, Nx, precision="mixed")
    assert _rel(d(th, ph, w), ref) <= 1e-9
    th, ph, w = _full_sky(50000, 4, wkind="normal")
    a = d(th, ph, w)
    d.set_precision("mixed_f64_tables")
    assert _rel(a, d(th, ph, w)) <= 1e-8


@pytest.mark.parametrize("nmaps", [1, 3, 8, 9, 17])
def test_maps_in_tensor_core_passes(nmaps):
    """Passes of up to eight maps per table read: every map equals its single-map call."""
    Nl, Nx, N = 96, 192, 40000
    rng = np.random.default_rng(nmaps)
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    W = rng.normal(1.0, 0.3, (nmaps, N))
    d = DirectSHT(Nl, Nx, precision="mixed")
    A = d.call_maps(th, ph, W)
    ref64 = DirectSHT(Nl, Nx)
    for k in range(nmaps):
        assert _rel(A[k], d(th, ph, W[k])) <= 1e-7, k
        assert _rel(A[k], ref64(th, ph, W[k])) <= 1e-7, k


def test_batch_of_point_sets_in_one_pass():
    Nl, Nx = 80, 160
    sets = [_full_sky(n, 100 + i) for i, n in enumerate([30000, 500, 12000, 64000, 2000])]
    d = DirectSHT(Nl, Nx, precision="mixed")
    got = d.call_batch(sets)
    tab = O.build_tables(Nl, Nx)
    for i, (th, ph, w) in enumerate(sets):
        assert _rel(got[i], O.direct_sht(tab, th, ph, w)) <= 1e-7, i


def test_compact_plan_nx_not_multiple_of_32():
    """K = 2 Nx padded to 64-byte rows, nodes not a multiple of the fold block."""
    Nl, Nx, N = 70, 77, 20000
    th, ph, w = _full_sky(N, 9)
    d = DirectSHT(Nl, Nx, compact_tables=True)
    assert _rel(d(th, ph, w), O.direct_sht(O.build_tables(Nl, Nx), th, ph, w)) <= 1e-7
