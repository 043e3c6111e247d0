"""Multi-map transforms (one point set, many weight maps) through dsht_execute_maps.

Every map must give the alm of a single-map call with the same points (the reference's
users loop DirectSHT.__call__ over maps, sht/sht.py:112-150).  FP64: within 1e-12 x
max|alm| of the oracle; mixed levels: within 1e-7 x max|alm| of the oracle."""
import numpy as np
import pytest
import torch

from directsht_b200 import DirectSHT
from oracle import dsht_oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _points(N, seed):
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    return rng, th, ph


@pytest.mark.parametrize("Nl,Nx,N,nmaps", [(64, 128, 20000, 5), (37, 50, 700, 3), (96, 192, 50000, 2)])
def test_maps_fp64_vs_oracle(Nl, Nx, N, nmaps):
    rng, th, ph = _points(N, 11 + Nl)
    W = rng.normal(1.0, 0.3, (nmaps, N))
    d = DirectSHT(Nl, Nx)
    A = d.call_maps(th, ph, W)
    assert A.shape == (nmaps, d.Nlm) and A.dtype == np.complex128
    tab = O.build_tables(Nl, Nx)
    for k in range(nmaps):
        ref = O.direct_sht(tab, th, ph, W[k])
        assert _rel(A[k], ref) <= 1e-12, k


def test_maps_f32_weights_are_exact():
    """float32 maps give the alm of their exact float64 widening."""
    Nl, Nx, N = 64, 128, 30000
    rng, th, ph = _points(N, 3)
    W = rng.normal(1.0, 0.3, (4, N)).astype(np.float32)
    d = DirectSHT(Nl, Nx)
    A = d.call_maps(th, ph, W)
    tab = O.build_tables(Nl, Nx)
    for k in range(4):
        assert _rel(A[k], O.direct_sht(tab, th, ph, W[k].astype(np.float64))) <= 1e-12


def test_maps_strided_torch_input_stays_on_device():
    Nl, Nx, N = 48, 96, 10000
    rng, th, ph = _points(N, 5)
    big = torch.tensor(rng.normal(1.0, 0.3, (3, N + 17)), device="cuda")
    W = big[:, :N]  # row stride N + 17
    d = DirectSHT(Nl, Nx)
    A = d.call_maps(torch.tensor(th, device="cuda"), torch.tensor(ph, device="cuda"), W)
    assert A.is_cuda and A.shape == (3, d.Nlm)
    for k in range(3):
        single = d(th, ph, W[k].cpu().numpy())
        assert _rel(A[k].cpu().numpy(), single) <= 1e-13


@pytest.mark.parametrize("precision", ["mixed", "mixed_f64_tables"])
def test_maps_mixed_vs_oracle(precision):
    Nl, Nx, N, nmaps = 128, 256, 200000, 3
    rng, th, ph = _points(N, 21)
    W = rng.normal(1.0, 0.3, (nmaps, N)).astype(np.float32)
    d = DirectSHT(Nl, Nx, precision=precision)
    A = d.call_maps(th, ph, W)
    tab = O.build_tables(Nl, Nx)
    for k in range(nmaps):
        ref = O.direct_sht(tab, th, ph, W[k].astype(np.float64))
        assert _rel(A[k], ref) <= 1e-7, (k, _rel(A[k], ref))


def test_single_map_f32_and_one_row():
    Nl, Nx, N = 32, 64, 5000
    rng, th, ph = _points(N, 8)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(Nl, Nx)
    A = d.call_maps(th, ph, w)  # 1-D weights: one map
    assert A.shape == (1, d.Nlm)
    assert _rel(A[0], d(th, ph, w)) <= 1e-13


def test_maps_empty_and_polar_failure():
    d = DirectSHT(16, 32)
    A = d.call_maps(np.zeros(0), np.zeros(0), np.zeros((2, 0)))
    assert A.shape == (2, d.Nlm) and not np.any(A)
    # xmax below sin(pi/4): cos(theta) = 0.7 at phi = 0 maps to cos(theta') = -sin(theta) = -0.714 after the rotation.
    d2 = DirectSHT(16, 32, xmax=0.6)
    th = np.array([np.arccos(0.7), 1.5])
    ph = np.array([0.0, 0.2])
    A2 = d2.call_maps(th, ph, np.ones((2, 2)))
    assert not np.any(A2)


def test_maps_per_pass_does_not_change_results():
    """The bin sums of a map do not depend on the grouping of maps into contraction passes,
    and the contraction's integer sums are exact, so every map's alm is bit for bit the
    same for every grouping."""
    Nl, Nx, N = 96, 192, 60000
    rng, th, ph = _points(N, 31)
    W = rng.normal(1.0, 0.3, (5, N)).astype(np.float32)
    d = DirectSHT(Nl, Nx, precision="mixed")
    out = []
    for per_pass in (1, 2, 3, 4):
        assert d.tune(maps_per_pass=per_pass)["maps_per_pass"] == per_pass
        out.append(d.call_maps(th, ph, W))
    assert all(np.array_equal(out[0], o) for o in out[1:])
    ref = O.direct_sht(O.build_tables(Nl, Nx), th, ph, W[4].astype(np.float64))
    assert _rel(out[0][4], ref) <= 1e-7


@pytest.mark.parametrize("piece", [256, 512, 2048])
def test_piece_size_tuning(piece):
    Nl, Nx, N = 64, 64, 40000  # few bins: many points per bin, split into pieces
    rng, th, ph = _points(N, 41)
    w = rng.uniform(0.5, 1.5, N)
    ref = O.direct_sht(O.build_tables(Nl, Nx), th, ph, w)
    d = DirectSHT(Nl, Nx)
    d.tune(piece_max=piece)
    assert _rel(d(th, ph, w), ref) <= 1e-12
    d.set_precision("mixed_f64_tables")
    assert _rel(d(th, ph, w), ref) <= 1e-7


def test_tune_rejects_bad_values():
    from directsht_b200 import _lib as L
    d = DirectSHT(16, 32)
    for param, value in ((L.DSHT_TUNE_PIECE_MAX, 100), (L.DSHT_TUNE_PIECE_MAX, 70000),
                         (L.DSHT_TUNE_PIECE_MAX, 4100), (L.DSHT_TUNE_MAPS_PER_PASS, 9),
                         (L.DSHT_TUNE_BIN_SUMS, 4), (L.DSHT_TUNE_BIN_SUMS, -1), (77, 1)):
        assert d._lib.dsht_plan_tune(d._plan, param, value) == L.DSHT_ERR_INVALID
    assert d.tune() == {"piece_max": 0, "maps_per_pass": 0, "bin_sums": "auto"}


@pytest.mark.slow
def test_maps_c3_scale_columns_vs_oracle():
    """The multi-map workload at full size: Nl=1024, Nx=2048, 2e6 full-sky points, 64 float32
    maps w ~ N(1, 0.3^2), mixed level.  Maps 0, 31 and 63 against the per-m oracle on both
    point sets (equatorial, and polar points rotated by 90 degrees), and the whole __call__
    against the sum of the parts (the rotation kernel is pinned to the oracle elsewhere)."""
    import ctypes as ct
    from directsht_b200 import _lib as L
    Nl, Nx, N, nmaps = 1024, 2048, 2_000_000, 64
    rng, th, ph = _points(N, 0)
    W = rng.normal(1.0, 0.3, (nmaps, N)).astype(np.float32)
    d = DirectSHT(Nl, Nx, precision="mixed")
    full = d.call_maps(th, ph, W)
    pol = np.abs(np.cos(th)) >= 0.75
    equ = ~pol
    tr, pr = O.rotate_points(th[pol], ph[pol])
    a_equ = d.call_maps(th[equ], ph[equ], np.ascontiguousarray(W[:, equ]), mode="basic")
    a_rot = d.call_maps(tr, pr, np.ascontiguousarray(W[:, pol]), mode="basic")
    for k in (0, 31, 63):
        scale = np.abs(full[k]).max()
        for a, (t_, p_, w_) in ((a_equ, (th[equ], ph[equ], W[k, equ])), (a_rot, (tr, pr, W[k, pol]))):
            for m in (0, 1, 511, 1023):
                r0 = O.healpy_index(m, m, Nl)
                col = O.basic_sht_column(Nl, Nx, 0.75, m, t_, p_, w_.astype(np.float64))
                assert np.abs(a[k, r0:r0 + Nl - m] - col).max() <= 1e-7 * np.abs(a[k]).max(), (k, m)
        rot = torch.from_numpy(a_rot[k]).cuda()
        back = torch.empty_like(rot)
        L.check(d._lib.dsht_rotate_back(d._plan, L.ptr(rot), None, L.ptr(back), None))
        torch.cuda.synchronize()
        assert np.abs(full[k] - (a_equ[k] + back.cpu().numpy())).max() <= 1e-7 * scale, k
