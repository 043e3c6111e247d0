"""GPU parity tests: the CUDA path through the C ABI against the oracle and the
reference's golden vectors.  Tolerance for the plain FP64 path: 1e-12 x max|alm|."""
import ctypes as ct

import numpy as np
import pytest
import torch

import inputs as I
from directsht_b200 import DirectSHT
from directsht_b200 import _lib as L
from oracle import dsht_oracle as O
from oracle import ref_csht

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _golden(name):
    return np.load(f"{I.__file__.rsplit('/', 1)[0]}/{name}.npz")


def test_tables_match_reference_rows():
    g = _golden("tables_nl500_nx1024")
    d = DirectSHT(int(g["Nl"]), int(g["Nx"]), float(g["xmax"]))
    assert np.array_equal(d.x, g["x"])
    worst = 0.0
    for n, (l, m) in enumerate(g["rows"]):
        yv, yd = d.get_Ylm(l, m)[g["ix"]], d.get_dYlm(l, m)[g["ix"]]
        worst = max(worst, _rel(yv, g["yv"][n]) if np.any(g["yv"][n]) else 0.0,
                    _rel(yd, g["yd"][n]) if np.any(g["yd"][n]) else 0.0)
    for n, (l, m) in enumerate(g["full_rows"]):
        worst = max(worst, _rel(d.get_Ylm(l, m), g["yv_full"][n]), _rel(d.get_dYlm(l, m), g["yd_full"][n]))
    assert worst <= 1e-14, worst


def test_full_tables_match_oracle():
    Nl, Nx = 70, 131
    d = DirectSHT(Nl, Nx)
    tab = O.build_tables(Nl, Nx)
    assert _rel(d.Yv, tab.Yv) <= 1e-14
    assert _rel(d.Yd, tab.Yd) <= 1e-14


@pytest.mark.parametrize("compact", [False, True])
def test_jax_layout_tables(compact):
    """Yv/Yd in the JAX path's [m, l-m, :] layout with the unphysical entries nulled
    (sht/legendre_jax.py:14-25): the same rows as the Healpy-order tables, host and device."""
    Nl, Nx = 70, 132
    d = DirectSHT(Nl, Nx, table_layout="jax", compact_tables=compact)
    tab = O.build_tables(Nl, Nx)
    for which, ref, host in (("Yv", tab.Yv, d.Yv), ("Yd", tab.Yd, d.Yd)):
        assert host.shape == (Nl, Nl, Nx)
        dev = d.table_on_device(which).cpu().numpy()
        assert np.array_equal(dev, host)
        tol = 1e-7 if compact else 1e-14
        for m in range(Nl):
            r0 = O.healpy_index(m, m, Nl)
            assert _rel(host[m, :Nl - m], ref[r0:r0 + Nl - m]) <= tol, (which, m)
            assert not np.any(host[m, Nl - m:])
    # get_Ylm is layout independent (sht/sht.py:69-93)
    assert np.array_equal(d.get_Ylm(5, 3), d.Yv[3, 2])


@pytest.mark.parametrize("name", list(I.CASES))
def test_golden_cases(name):
    s = I.CASES[name]
    g = _golden(name)
    th, ph, w = I.make_inputs(name)
    d = DirectSHT(s["Nl"], s["Nx"], s.get("xmax", 0.75))
    if s["entry"] == "call":
        a = d(th, ph, w)
    else:
        a = d.basic_sht(th, ph, w.copy(), reg_factor=s.get("reg", 1.0), verbose=False)
    assert a.dtype == np.complex128 and a.shape == (d.Nlm,)
    assert _rel(a, g["alm"]) <= TOL_FP64
    np.testing.assert_allclose(d.alm2cl(a), g["cl"], rtol=1e-10, atol=1e-13 * np.abs(g["alm"]).max() ** 2)


@pytest.mark.parametrize("name", ["c1_full_sky", "small_call", "cap_c2like", "single_point", "xmax_0p8"])
def test_alm2cl_on_device_matches_reference_golden(name):
    """DirectSHT.alm2cl of device alm (dsht_alm2cl_device) against the cl the reference's own
    alm2cl (sht/sht.py:95-109) produced for the same case; the alm never leave the GPU."""
    s = I.CASES[name]
    g = _golden(name)
    th, ph, w = I.make_inputs(name)
    d = DirectSHT(s["Nl"], s["Nx"], s.get("xmax", 0.75))
    dev = [torch.from_numpy(x).cuda() for x in (th, ph, w)]
    if s["entry"] == "call":
        a = d(*dev)
    else:
        a = d.basic_sht(dev[0], dev[1], dev[2].clone(), reg_factor=s.get("reg", 1.0), verbose=False)
    assert a.is_cuda
    cl = d.alm2cl(a)
    assert cl.is_cuda and cl.dtype == torch.float64 and cl.shape == (d.Nell,)
    scale = np.abs(g["alm"]).max() ** 2
    np.testing.assert_allclose(cl.cpu().numpy(), g["cl"], rtol=1e-10, atol=1e-13 * scale)
    # several maps at once: rows of a (nmaps, Nlm) tensor, each the single-map spectrum
    two = torch.stack([a, 2.0 * a])
    cl2 = d.alm2cl(two).cpu().numpy()
    np.testing.assert_allclose(cl2[0], cl.cpu().numpy(), rtol=1e-15, atol=0)
    np.testing.assert_allclose(cl2[1], 4.0 * cl.cpu().numpy(), rtol=1e-14, atol=0)


@pytest.mark.parametrize("Nl,Nx,N,seed", [(1, 2, 10, 0), (2, 3, 50, 1), (3, 5, 1, 2), (37, 50, 1000, 3),
                                          (64, 128, 30000, 4), (129, 64, 5000, 5), (200, 300, 20000, 6)])
def test_random_full_sky_vs_oracle(Nl, Nx, N, seed):
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.lognormal(0, 0.5, N)
    a = DirectSHT(Nl, Nx)(th, ph, w)
    ref = O.direct_sht(O.build_tables(Nl, Nx), th, ph, w)
    assert _rel(a, ref) <= TOL_FP64


def test_many_points_in_one_bin_split_into_pieces():
    rng = np.random.default_rng(7)
    N = 60000
    th = np.arccos(rng.uniform(0.40, 0.401, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(96, 64)
    a = d.basic_sht(th, ph, w, verbose=False)
    ref = O.basic_sht(O.build_tables(96, 64), th, ph, w)
    assert _rel(a, ref) <= TOL_FP64


def test_device_tensors_in_and_out():
    rng = np.random.default_rng(8)
    N = 4000
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(48, 96)
    a_host = d(th, ph, w)
    dev = [torch.from_numpy(v).cuda() for v in (th, ph, w)]
    a_dev = d(*dev)
    assert isinstance(a_dev, torch.Tensor) and a_dev.is_cuda and a_dev.dtype == torch.complex128
    assert np.array_equal(a_dev.cpu().numpy(), a_host) or _rel(a_dev.cpu().numpy(), a_host) <= 1e-15


def test_host_entry_point_matches_device_entry_point():
    rng = np.random.default_rng(9)
    N = 5000
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    d = DirectSHT(40, 80)
    out = np.zeros(d.Nlm, dtype=np.complex128)
    L.check(d._lib.dsht_execute_host(d._plan, L.dptr(th), L.dptr(ph), L.dptr(w), N, L.DSHT_MODE_CALL,
                                     out.view(np.float64).ctypes.data_as(ct.POINTER(ct.c_double))))
    assert _rel(out, d(th, ph, w)) <= 1e-15


# ---- error behaviour mirrors the reference ------------------------------------------
def test_basic_sht_rejects_polar_theta():
    d = DirectSHT(16, 32)
    with pytest.raises(AssertionError, match="theta must be in"):
        d.basic_sht(np.array([0.1, 1.5]), np.array([0.0, 1.0]), np.ones(2), verbose=False)


def test_basic_sht_rejects_empty():
    d = DirectSHT(16, 32)
    with pytest.raises(ValueError, match="empty"):
        d.basic_sht(np.array([]), np.array([]), np.array([]), verbose=False)


def test_call_on_no_points_is_zero():
    d = DirectSHT(16, 32)
    a = d(np.array([]), np.array([]), np.array([]))
    assert a.shape == (d.Nlm,) and not np.any(a)


def test_length_mismatch():
    d = DirectSHT(16, 32)
    with pytest.raises(AssertionError, match="same length"):
        d(np.ones(3), np.ones(2), np.ones(3))


def test_nan_theta_is_dropped_like_the_reference():
    rng = np.random.default_rng(10)
    N = 3000
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    th_nan = th.copy()
    th_nan[::7] = np.nan
    d = DirectSHT(32, 64)
    keep = ~np.isnan(th_nan)
    assert _rel(d(th_nan, ph, w), d(th[keep], ph[keep], w[keep])) <= 1e-15


def test_small_xmax_polar_failure_returns_zeros(capsys):
    rng = np.random.default_rng(12)
    th = np.arccos(rng.uniform(-1, 1, 2000))
    ph = rng.uniform(0, 2 * np.pi, 2000)
    d = DirectSHT(16, 32, xmax=0.6)
    a = d(th, ph, np.ones(2000))
    assert not np.any(a)
    assert "xmax is smaller than sin(pi/4)" in capsys.readouterr().out


def test_basic_sht_scales_weights_in_place():
    rng = np.random.default_rng(13)
    th = np.arccos(rng.uniform(-0.7, 0.7, 300))
    ph = rng.uniform(0, 2 * np.pi, 300)
    w = rng.uniform(0.5, 1.5, 300)
    w0 = w.copy()
    d = DirectSHT(12, 24)
    a = d.basic_sht(th, ph, w, reg_factor=4.0, verbose=False)
    np.testing.assert_array_equal(w, 4.0 * w0)
    assert _rel(a, O.basic_sht(O.build_tables(12, 24), th, ph, w0)) <= TOL_FP64


# ---- drop-ins for the reference's ctypes library ---------------------------------------
def test_make_table_drop_in():
    lib = L.load()
    Nl, Nx = 30, 60
    Nlm = Nl * (Nl + 1) // 2
    Yv = np.zeros(Nlm * Nx)
    Yd = np.zeros(Nlm * Nx)
    assert lib.dsht_make_table(Nl, Nx, 0.75, L.dptr(Yv), L.dptr(Yd)) == 0
    tab = O.build_tables(Nl, Nx)
    assert _rel(Yv.reshape(Nlm, Nx), tab.Yv) <= 1e-14
    assert _rel(Yd.reshape(Nlm, Nx), tab.Yd) <= 1e-14


@pytest.mark.skipif(not ref_csht.available(), reason="oracle/_ref not built")
def test_do_transform_drop_in_matches_reference_c():
    lib = L.load()
    Nl, Nx, N = 48, 96, 4000
    rng = np.random.default_rng(14)
    cost = np.sort(rng.uniform(0.0, 0.74, N))
    phi = rng.uniform(0, 2 * np.pi, N)
    wt = rng.uniform(0.5, 1.5, N)
    Nlm = Nl * (Nl + 1) // 2
    carr, sarr = np.zeros(Nlm), np.zeros(Nlm)
    dummy = np.zeros(1)
    assert lib.dsht_do_transform(Nl, Nx, 0.75, L.dptr(dummy), L.dptr(dummy), N, L.dptr(cost), L.dptr(phi),
                                 L.dptr(wt), L.dptr(carr), L.dptr(sarr)) == 0
    r = ref_csht.RefCSHT(Nl, Nx)
    cref, sref = np.zeros(Nlm), np.zeros(Nlm)
    r.lib.do_transform(Nl, Nx, 0.75, ref_csht._p(r.Yv), ref_csht._p(r.Yd), N, ref_csht._p(cost),
                       ref_csht._p(phi), ref_csht._p(wt), ref_csht._p(cref), ref_csht._p(sref))
    scale = max(np.abs(cref).max(), np.abs(sref).max())
    assert np.abs(carr - cref).max() <= 1e-12 * scale
    assert np.abs(sarr - sref).max() <= 1e-12 * scale


# ---- full size: survey-like single map (Nl=1024, Nx=2048, N=1e7) ------------------------
def _c2_points(N, seed=0):
    rng = np.random.default_rng(seed)
    th = np.arccos(rng.uniform(np.cos(1.2), np.cos(0.3), N))
    ph = rng.uniform(0, 1.5 * np.pi, N)
    w = rng.lognormal(0.0, 0.5, N)
    return th, ph, w


@pytest.mark.slow
def test_c2_full_size_columns_and_rotation():
    Nl, Nx, N = 1024, 2048, 10_000_000
    th, ph, w = _c2_points(N)
    d = DirectSHT(Nl, Nx)
    full = d(th, ph, w)
    pol = np.abs(np.cos(th)) >= 0.75
    equ = ~pol
    a_equ = d.basic_sht(th[equ], ph[equ], w[equ].copy(), verbose=False)
    tr, pr = O.rotate_points(th[pol], ph[pol])
    a_rot = d.basic_sht(tr, pr, w[pol].copy(), verbose=False)
    scale = np.abs(full).max()
    # columns of both basic transforms against the per-m oracle
    for m in (0, 1, 2, 511, 1000, 1023):
        r0 = O.healpy_index(m, m, Nl)
        for a, (t_, p_, w_) in ((a_equ, (th[equ], ph[equ], w[equ])), (a_rot, (tr, pr, w[pol]))):
            col = O.basic_sht_column(Nl, Nx, 0.75, m, t_, p_, w_)
            assert np.abs(a[r0:r0 + Nl - m] - col).max() <= TOL_FP64 * np.abs(a).max(), m
    # the rotation kernel against the oracle's Wigner-d restatement
    ad = torch.from_numpy(a_rot).cuda()
    out = torch.empty_like(ad)
    L.check(d._lib.dsht_rotate_back(d._plan, L.ptr(ad), None, L.ptr(out), None))
    torch.cuda.synchronize()
    back = out.cpu().numpy()
    assert _rel(back, O.rotate_alm_back(a_rot, Nl)) <= TOL_FP64
    # and the fused __call__ is the sum of the two
    assert np.abs(full - (a_equ + back)).max() <= TOL_FP64 * scale
    # size-independent property: rotating the equatorial points about z by alpha
    # multiplies a_lm by exp(-i m alpha)
    alpha = 0.37
    a_shift = d.basic_sht(th[equ], np.mod(ph[equ] + alpha, 2 * np.pi), w[equ].copy(), verbose=False)
    _, ms = O.getlm(Nl)
    assert np.abs(a_shift - a_equ * np.exp(-1j * ms * alpha)).max() <= TOL_FP64 * np.abs(a_equ).max()
