"""The NUFFT bin sums of the mixed levels (nufft.cu) against the FP64 path and the oracle.

The mixed levels form each bin's sums v_k[m] = sum_p g_k(p) e^{i m phi_p} by a type-1
non-uniform FFT (spread onto a 4 x 2^ceil(log2 Nl)-cell grid with a width-12 kernel, FFT,
deconvolution), error about 5e-12 of the bin's sum |g_k|.  With the FP64 tables in the
contraction (mixed_f64_tables) that is the only approximation, so those results must agree
with the plain FP64 transform to 1e-10 of max|alm|; with the digit tables (mixed) to 1e-8.
The spread adds 64-bit fixed-point values with integer atomics, so results are bitwise
repeatable.  The direct tensor-core sums stay selectable (tune(bin_sums='tc')); AUTO picks
by the average number of points per bin key."""
import numpy as np
import pytest

from directsht_b200 import DirectSHT
from oracle import dsht_oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def _sky(N, seed, wkind="lognormal"):
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = {"lognormal": lambda: rng.lognormal(0, 0.5, N), "normal": lambda: rng.normal(0, 1, N),
         "wide": lambda: rng.lognormal(0, 3.0, N)}[wkind]()
    return th, ph, w


# Nl = 1 .. 2048: grids of 64 .. 8192 cells, one and two FFT passes per piece (Nl > 1024)
@pytest.mark.parametrize("Nl,Nx,N", [(1, 8, 5000), (7, 16, 3000), (64, 128, 40000), (500, 1024, 200000),
                                     (1000, 2000, 300000), (1025, 2050, 200000), (2048, 4096, 150000)])
def test_nufft_bin_sums_vs_fp64(Nl, Nx, N):
    th, ph, w = _sky(N, Nl)
    d = DirectSHT(Nl, Nx)
    ref = d(th, ph, w)
    d.set_precision("mixed_f64_tables")
    assert d.tune()["bin_sums"] == "auto"
    assert d.tune(bin_sums="nufft")["bin_sums"] == "nufft"
    a = d(th, ph, w)
    assert _rel(a, ref) <= 1e-10
    assert np.array_equal(a, d(th, ph, w))  # integer spreading: bitwise repeatable
    d.set_precision("mixed")
    assert _rel(d(th, ph, w), ref) <= 1e-8


def test_nufft_vs_oracle_and_tensor_core_sums():
    """Both bin-sum methods against the oracle on the same points; the NUFFT one is the
    closer by orders of magnitude."""
    Nl, Nx, N = 200, 400, 100000
    th, ph, w = _sky(N, 5)
    ref = O.direct_sht(O.build_tables(Nl, Nx), th, ph, w)
    d = DirectSHT(Nl, Nx, precision="mixed_f64_tables")
    d.tune(bin_sums="nufft")
    e_nufft = _rel(d(th, ph, w), ref)
    assert d.tune(bin_sums="tc")["bin_sums"] == "tc"
    e_tc = _rel(d(th, ph, w), ref)
    assert e_nufft <= 1e-10 and e_tc <= 1e-7 and e_nufft < e_tc / 100
    assert d.tune(bin_sums="nufft")["bin_sums"] == "nufft"
    assert _rel(d(th, ph, w), ref) == e_nufft


@pytest.mark.parametrize("wkind", ["normal", "wide"])
def test_nufft_weights_without_the_fixed_point_limits(wkind):
    """Zero-mean weights (sums cancel) and lognormal sigma = 3 weights (many decades): the
    direct tensor-core sums lose accuracy on both (their scale is a piece's largest |w|);
    the NUFFT sums do not."""
    Nl, Nx, N = 128, 256, 120000
    th, ph, w = _sky(N, 11, wkind)
    d = DirectSHT(Nl, Nx)
    ref = d(th, ph, w)
    d.set_precision("mixed_f64_tables")
    d.tune(bin_sums="nufft")
    assert _rel(d(th, ph, w), ref) <= (1e-9 if wkind == "normal" else 1e-10)


@pytest.mark.parametrize("piece", [256, 2048, 16384, 65536])
def test_nufft_piece_sizes_and_heavy_bins(piece):
    """A polar cap of radius 0.05: every point in a handful of bins, so bins split into many
    pieces (each its own FFT) or fill one; results agree whatever the piece size."""
    rng = np.random.default_rng(piece)
    N, Nl, Nx = 300000, 256, 512
    th = np.arccos(rng.uniform(np.cos(0.05), 1.0, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(Nl, Nx)
    ref = d(th, ph, w)
    d.set_precision("mixed_f64_tables")
    d.tune(piece_max=piece, bin_sums="nufft")
    assert _rel(d(th, ph, w), ref) <= 1e-10


def test_nufft_many_maps_match_single_calls():
    Nl, Nx, N = 96, 192, 50000
    th, ph, _ = _sky(N, 21)
    W = np.random.default_rng(22).normal(1.0, 0.3, (5, N))
    d = DirectSHT(Nl, Nx, precision="mixed")
    d.tune(bin_sums="nufft")
    A = d.call_maps(th, ph, W)
    for k in range(5):
        assert _rel(A[k], d(th, ph, W[k])) <= 1e-12


def test_auto_bin_sums_follow_points_per_key():
    """AUTO takes the NUFFT sums from 512 points per bin key on average, the FP64 direct sums
    below 28 and the tensor-core sums in between: each call here agrees with its forced
    method (bit for bit for the NUFFT and tensor-core sums, whose per-piece sums are exact
    integers when pieces of up to 2048 points keep every bin one piece; to FP64 rounding for
    the FP64 sums, whose order of adds follows the sort) and not with the tensor-core sums."""
    Nl, Nx = 64, 32  # 4 x 31 = 124 keys: the NUFFT from 63488 points, FP64 below 3472
    th, ph, w = _sky(100000, 31)
    d = DirectSHT(Nl, Nx, precision="mixed")
    d.tune(piece_max=2048)
    for N, method in ((100000, "nufft"), (20000, "tc")):
        a = d(th[:N], ph[:N], w[:N])
        d.tune(bin_sums=method)
        assert np.array_equal(a, d(th[:N], ph[:N], w[:N])), (N, method)
        d.tune(bin_sums="auto")
    N = 2500
    a = d(th[:N], ph[:N], w[:N])
    d.tune(bin_sums="fp64")
    a64 = d(th[:N], ph[:N], w[:N])
    d.tune(bin_sums="tc")
    atc = d(th[:N], ph[:N], w[:N])
    d.tune(bin_sums="auto")
    scale = np.abs(a64).max()
    assert np.abs(a - a64).max() <= 1e-13 * scale
    assert np.abs(a - atc).max() > 1e-11 * scale


def test_batch_items_choose_their_own_bin_sums():
    """In a batch call each transform takes the bin-sum method its own size selects (not the
    one of the batch's largest transform).  With pieces of up to 2048 points every bin here
    is one piece and each item equals the same transform run alone to FP64 rounding; with the
    default piece sizes (a workspace laid out for the NUFFT's large pieces, smaller pieces
    for the direct sums of the smaller items) each item agrees with it within the mixed
    tolerance (pieces cut from the sort's order quantise differently)."""
    Nl, Nx = 64, 32  # 124 keys: NUFFT from 63488 points, FP64 sums below 3472
    th, ph, w = _sky(100000, 37)
    d = DirectSHT(Nl, Nx, precision="mixed")
    sets = [(th[:N], ph[:N], w[:N]) for N in (100000, 20000, 2500)]
    for piece, tol in ((2048, 1e-12), (0, 1e-8)):
        d.tune(piece_max=piece)
        batch = d.call_batch(sets)
        for (t, p, ww), a in zip(sets, batch):
            alone = d(t, p, ww)
            assert np.abs(a - alone).max() <= tol * np.abs(alone).max(), (piece, len(t))
