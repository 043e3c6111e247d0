"""The NUFFT bin sums' arithmetic on the CPU (no GPU): the library's own host tables (kernel
polynomials, 1/Psi(m), grid size) driving a numpy restatement of what nufft_sums_kernel
does -- 46-bit fixed-point spread of the four Hermite weights onto a periodic real grid of
n cells, two real grids per complex FFT, the conjugate-symmetry split and the division by
Psi(m) -- against the direct sums v_k[m] = sum_p g_k(p) e^{i m phi_p}
(sht/shared_interp_funcs.py:88-105).  The same split words (low 16 bits, high bits) are
summed as the kernel's reductions sum them."""
import ctypes as ct

import numpy as np
import pytest

from directsht_b200 import _lib as L

W, DEG = 12, 11


def _tables(Nl):
    lib = L.load()
    logn = ct.c_int()
    poly = np.zeros(W * (DEG + 1))
    dinv = np.zeros(Nl)
    L.check(lib.dsht_test_nufft_tables(Nl, ct.byref(logn), L.dptr(poly), L.dptr(dinv)))
    return logn.value, poly.reshape(W, DEG + 1), dinv


def _hermite(t, w):
    return np.stack([w * ((2 * t + 1) * (1 - t) ** 2), w * (t * (1 - t) ** 2),
                     w * (t ** 2 * (3 - 2 * t)), w * (t ** 2 * (t - 1))])


def _nufft_model(phi, t, w, Nl):
    logn, poly, dinv = _tables(Nl)
    n = 1 << logn
    u = phi * (n / (2 * np.pi))
    fl = np.floor(u)
    s = 2 * (u - fl) - 1
    cb = fl.astype(np.int64) - W // 2 + 1
    ker = np.zeros((W, len(phi)))
    for i in range(W):
        acc = np.full(len(phi), poly[i, DEG])
        for d in range(DEG - 1, -1, -1):
            acc = acc * s + poly[i, d]
        ker[i] = acc
    g = _hermite(t, w)
    wsum = np.abs(w).sum() * (1 + len(w) * 2.0 ** -52)
    e = int(np.frexp(wsum)[1])
    scale, step = 2.0 ** (46 - e), 2.0 ** (e - 46)
    # per grid: low-16-bit and high sums of the rounded fixed-point values, as integers
    lo = np.zeros((4, n), np.int64)
    hi = np.zeros((4, n), np.int64)
    for i in range(W):
        cell = (cb + i) & (n - 1)
        for k in range(4):
            X = np.rint(g[k] * scale * ker[i]).astype(np.int64)
            assert np.abs(X).max() < 2 ** 47
            np.add.at(lo[k], cell, X & 0xFFFF)
            np.add.at(hi[k], cell, X >> 16)
    assert lo.max() < 2 ** 32 and np.abs(hi).max() < 2 ** 31
    G = (hi * 65536 + lo).astype(np.float64)
    out = np.zeros((8, Nl))
    m = np.arange(Nl)
    for pair in range(2):
        Z = np.fft.ifft(G[2 * pair] + 1j * G[2 * pair + 1]) * n  # sum_j z_j e^{+2 pi i m j / n}
        a, b = Z[m], Z[(n - m) & (n - 1)]
        di = 0.5 * step * dinv
        out[4 * pair + 0] = (a.real + b.real) * di
        out[4 * pair + 1] = (a.imag - b.imag) * di
        out[4 * pair + 2] = (a.imag + b.imag) * di
        out[4 * pair + 3] = (b.real - a.real) * di
    return out, g


@pytest.mark.parametrize("Nl,npts,wkind", [(64, 300, "lognormal"), (1000, 2000, "lognormal"),
                                           (1024, 3000, "normal"), (2048, 1500, "wide")])
def test_nufft_arithmetic_vs_direct_sums(Nl, npts, wkind):
    rng = np.random.default_rng(Nl + npts)
    phi = rng.uniform(0, 2 * np.pi, npts)
    t = rng.uniform(0, 1, npts)
    w = {"lognormal": rng.lognormal(0, 0.5, npts), "normal": rng.normal(0, 1, npts),
         "wide": rng.lognormal(0, 3.0, npts)}[wkind]
    out, g = _nufft_model(phi, t, w, Nl)
    direct = g @ np.exp(1j * np.outer(phi, np.arange(Nl)))
    ref = np.zeros((8, Nl))
    ref[0::2], ref[1::2] = direct.real, direct.imag
    err = np.abs(out - ref).max() / np.abs(g).sum(axis=1).max()
    assert err <= 5e-11, err


def test_nufft_tables_shape():
    for Nl, logn in ((1, 7), (32, 7), (33, 8), (1000, 12), (1024, 12), (1025, 13), (2048, 13)):
        got, poly, dinv = _tables(Nl)
        assert got == logn, (Nl, got)
        assert np.all(np.isfinite(poly)) and np.all(dinv > 0)
    # the kernel's values at the cell of a point sitting on a cell (f = 0): psi(W/2 - 1 - i)
    _, poly, _ = _tables(64)
    at_f0 = poly @ ((-1.0) ** np.arange(DEG + 1))  # s = -1
    z = 2 * (W / 2 - 1 - np.arange(W)) / W
    psi = np.where(np.abs(z) < 1, np.exp(2.30 * W * (np.sqrt(np.clip(1 - z * z, 0, None)) - 1)), 0.0)
    assert np.abs(at_f0 - psi).max() <= 1e-11
