"""Mode coupling of pseudo-Cl (the reference's MaskDeconvolution, sht/mask_deconvolution.py).

CPU: the oracle's restatement of the reference's 3j recursion and of get_M against the
matrix the reference itself produced (tests/golden/mode_coupling.npz), and the closed form
against both.  GPU (marked): dsht_mode_coupling and directsht_b200.MaskDeconvolution against
the same golden values, the full-sky identity, and the closed form at Nl = 400."""
import numpy as np
import pytest

import inputs as I
from oracle import dsht_oracle as O


def _golden():
    return np.load(f"{I.__file__.rsplit('/', 1)[0]}/mode_coupling.npz")


def test_oracle_recursion_matches_reference_matrix():
    g = _golden()
    M = O.mode_coupling(int(g["Nl"]), g["W"])
    assert np.abs(M - g["Mll"]).max() <= 1e-14 * np.abs(g["Mll"]).max()


def test_closed_form_matches_recursion():
    g = _golden()
    M = O.mode_coupling_closed_form(int(g["Nl"]), g["W"])
    assert np.abs(M - g["Mll"]).max() <= 1e-12 * np.abs(g["Mll"]).max()


def test_threej_known_values():
    # (2 2 0; 000) = 1/sqrt(5); (1 1 2; 000) = sqrt(2/15); odd J vanishes
    assert abs(O.threej000(2, 2, 0) - 1 / np.sqrt(5)) < 1e-15
    assert abs(O.threej000(1, 1, 2) - np.sqrt(2 / 15)) < 1e-15
    assert O.threej000(1, 2, 2) == 0.0


@pytest.mark.gpu
def test_gpu_mode_coupling_matches_reference():
    from directsht_b200 import MaskDeconvolution
    from directsht_b200.mask import mode_coupling_matrix
    g = _golden()
    Nl = int(g["Nl"])
    M = mode_coupling_matrix(Nl, g["W"])
    assert np.abs(M - g["Mll"]).max() <= 1e-12 * np.abs(g["Mll"]).max()
    md = MaskDeconvolution(Nl, g["W"].copy(), verbose=False)
    assert np.abs(md.get_M(debug=True) - np.eye(Nl)).max() <= 1e-12
    np.testing.assert_array_equal(md.binning_matrix("linear", start=2, step=8), g["b_lin"])
    np.testing.assert_array_equal(md.binning_matrix("sqrt", start=2, step=4), g["b_sqrt"])
    for mode, e_ref, c_ref in (("deconvolution", g["ells_d"], g["Cb_d"]), ("normalization", g["ells_n"], g["Cb_n"])):
        ells, Cb = md(g["Cl"], g["b_lin"], mode=mode)
        np.testing.assert_allclose(ells, e_ref, rtol=1e-15)
        np.testing.assert_allclose(Cb, c_ref, rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(md.window_matrix(g["b_sqrt"], "deconvolution"), g["win_d"], rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(md.window_matrix(g["b_sqrt"], "normalization"), g["win_n"], rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_gpu_mode_coupling_large_vs_closed_form():
    from directsht_b200.mask import mode_coupling_matrix
    Nl = 400
    ell = np.arange(2 * Nl - 1)
    W = np.exp(-ell / 30.0) * (1.2 + np.sin(ell / 7.0))
    M = mode_coupling_matrix(Nl, W)
    rows = [0, 1, 57, 200, 399]
    ref = O.mode_coupling_closed_form(Nl, W)
    assert np.abs(M[rows] - ref[rows]).max() <= 1e-11 * np.abs(ref).max()
