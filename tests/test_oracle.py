"""CPU tests: the oracle against the reference's golden vectors and known answers."""
import numpy as np
import pytest

import inputs as I
from oracle import dsht_oracle as O
from oracle import ref_csht

GOLDEN = {name: spec for name, spec in I.CASES.items()}


def _golden(name):
    return np.load(f"{I.__file__.rsplit('/', 1)[0]}/{name}.npz")


def _oracle_alm(name):
    s = I.CASES[name]
    th, ph, w = I.make_inputs(name)
    tab = O.build_tables(s["Nl"], s["Nx"], s.get("xmax", 0.75))
    if s["entry"] == "call":
        return O.direct_sht(tab, th, ph, w)
    return O.basic_sht(tab, th, ph, w, reg_factor=s.get("reg", 1.0))


@pytest.mark.parametrize("name", [n for n in GOLDEN if n != "c1_full_sky"])
def test_oracle_matches_reference_golden(name):
    g = _golden(name)
    a = _oracle_alm(name)
    scale = np.abs(g["alm"]).max()
    assert np.abs(a - g["alm"]).max() <= 1e-13 * scale
    np.testing.assert_allclose(O.alm2cl(a, int(g["Nl"])), g["cl"], rtol=1e-11, atol=1e-14 * scale ** 2)


def test_oracle_matches_reference_c1():
    """Full sky, Nl=256, Nx=512, N=1e5, unit weights, seed 0, through the reference's __call__."""
    g = _golden("c1_full_sky")
    a = _oracle_alm("c1_full_sky")
    assert np.abs(a - g["alm"]).max() <= 1e-13 * np.abs(g["alm"]).max()


def test_tables_match_reference_rows():
    """Rows the reference's sht/test_sht.py inspects, from DirectSHT(500, 1024)."""
    g = _golden("tables_nl500_nx1024")
    Nl, Nx = int(g["Nl"]), int(g["Nx"])
    xx = O.x_grid(Nx, float(g["xmax"]))
    assert np.array_equal(xx, g["x"])
    rows = [tuple(r) for r in g["rows"]]
    by_m = {}
    for n, (l, m) in enumerate(rows):
        by_m.setdefault(m, []).append((n, l))
    for m, lst in by_m.items():
        P, D = O.table_column(Nl, xx, m)
        for n, l in lst:
            assert np.array_equal(P[l - m][g["ix"]], g["yv"][n]), (l, m)
            assert np.array_equal(D[l - m][g["ix"]], g["yd"][n]), (l, m)
    for n, (l, m) in enumerate(g["full_rows"]):
        P, D = O.table_column(Nl, xx, int(m))
        assert np.array_equal(P[l - m], g["yv_full"][n])
        assert np.array_equal(D[l - m], g["yd_full"][n])


def test_table_known_answers():
    """dY_20/dx = 3x sqrt(5/4pi), dY_10,10/dx = -5.42630291944221461 x (1-x^2)^4
    (sht/test_sht.py:57-59)."""
    tab = O.build_tables(16, 64)
    x = tab.x
    np.testing.assert_allclose(tab.Yd[O.healpy_index(2, 0, 16)], 3 * x * np.sqrt(5 / 4.0 / np.pi), rtol=1e-13,
                               atol=1e-15)
    np.testing.assert_allclose(tab.Yd[O.healpy_index(10, 10, 16)], -5.42630291944221461 * x * (1 - x ** 2) ** 4,
                               rtol=1e-12, atol=1e-15)


def test_tables_match_scipy():
    """Ylm(x, 0) against scipy's sph_harm_y for l < 45 (sht/test_sht.py:31-52)."""
    from scipy.special import sph_harm_y
    Nl, Nx = 45, 97
    tab = O.build_tables(Nl, Nx)
    th = np.arccos(tab.x)
    err = 0.0
    for ell in range(Nl):
        for m in range(ell + 1):
            ref = np.real(sph_harm_y(ell, m, th, 0.0))
            err = max(err, np.abs(tab.Yv[O.healpy_index(ell, m, Nl)] - ref).max())
    assert err < 1e-12


def test_table_column_matches_full_table():
    Nl, Nx = 33, 40
    tab = O.build_tables(Nl, Nx)
    for m in range(Nl):
        P, D = O.table_column(Nl, tab.x, m)
        r0 = O.healpy_index(m, m, Nl)
        assert np.array_equal(P, tab.Yv[r0:r0 + Nl - m])
        assert np.array_equal(D, tab.Yd[r0:r0 + Nl - m])


def test_basic_sht_column_matches_full():
    Nl, Nx = 30, 64
    tab = O.build_tables(Nl, Nx)
    rng = np.random.default_rng(11)
    th = np.arccos(rng.uniform(-0.74, 0.74, 2000))
    ph = rng.uniform(0, 2 * np.pi, 2000)
    w = rng.lognormal(0, 0.5, 2000)
    a = O.basic_sht(tab, th, ph, w)
    for m in (0, 1, 17, 29):
        r0 = O.healpy_index(m, m, Nl)
        c = O.basic_sht_column(Nl, Nx, 0.75, m, th, ph, w)
        assert np.abs(c - a[r0:r0 + Nl - m]).max() <= 1e-14 * np.abs(a).max()


@pytest.mark.parametrize("seed", [0, 1])
def test_rotation_matches_exact_definition(seed):
    """The healpy restatement: rotate points, transform exactly, rotate the alm back."""
    rng = np.random.default_rng(seed)
    N, Nl = 200, 14
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    exact = O.brute_force_alm(th, ph, w, Nl)
    t2, p2 = O.rotate_points(th, ph)
    back = O.rotate_alm_back(O.brute_force_alm(t2, p2, w, Nl), Nl)
    assert np.abs(back - exact).max() <= 1e-13 * np.abs(exact).max()
    # the rotated polar points land inside the table range
    pol = np.abs(np.cos(th)) >= 0.75
    assert np.all(np.abs(np.cos(t2[pol])) < 0.75)


@pytest.mark.parametrize("Nl", [1, 2, 5, 40, 97])
def test_precomputed_rotator_matches_rotate_alm_back(Nl):
    """AlmRotator (the CPU baseline's timed alm rotation) is rotate_alm_back regrouped."""
    rng = np.random.default_rng(Nl)
    Nlm = Nl * (Nl + 1) // 2
    a = rng.normal(size=Nlm) + 1j * rng.normal(size=Nlm)
    ref = O.rotate_alm_back(a, Nl)
    assert np.abs(O.AlmRotator(Nl)(a) - ref).max() <= 1e-14 * np.abs(ref).max()


def test_direct_sht_matches_exact_definition():
    """Spline error of the whole __call__ path against sum w conj(Y_lm)."""
    rng = np.random.default_rng(5)
    N, Nl = 500, 16
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    w = rng.uniform(0.5, 1.5, N)
    tab = O.build_tables(Nl, 512)
    a = O.direct_sht(tab, th, ph, w)
    exact = O.brute_force_alm(th, ph, w, Nl)
    assert np.abs(a - exact).max() <= 1e-8 * np.abs(exact).max()


@pytest.mark.parametrize("ell", [1, 7, 64, 511, 1023, 2047])
def test_wigner_d_columns_orthonormal(ell):
    D = O.wigner_d_halfpi_column(ell)  # d_{k,m}, k,m >= 0; d_{-k,m} = (-1)^(l-m) d_{k,m}
    norm = D[0] ** 2 + 2 * np.sum(D[1:] ** 2, axis=0)
    assert np.abs(norm - 1).max() < 1e-12
    # symmetry d_{k,m} = (-1)^(m-k) d_{m,k}
    k = np.arange(ell + 1)
    sign = (-1.0) ** (k[None, :] - k[:, None])
    assert np.abs(D - sign * D.T).max() < 1e-12


@pytest.mark.skipif(not ref_csht.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["small_call", "cap_c2like", "small_basic_mixed_sign", "xmax_0p8"])
def test_reference_c_path_matches_golden(name):
    """The reference's own C/OpenMP code (csht/sht_helper.c) agrees with its numpy path."""
    s = I.CASES[name]
    g = _golden(name)
    th, ph, w = I.make_inputs(name)
    r = ref_csht.RefCSHT(s["Nl"], s["Nx"], s.get("xmax", 0.75))
    a = r(th, ph, w) if s["entry"] == "call" else r.basic(th, ph, w)
    assert np.abs(a - g["alm"]).max() <= 1e-12 * np.abs(g["alm"]).max()
