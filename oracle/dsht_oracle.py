"""CPU oracle for the DirectSHT forward transform -- TEST INFRASTRUCTURE ONLY.

This module restates, in plain numpy, the algorithm of the reference's numpy/numba
path (martinjameswhite/directsht, ``sht/``) so that the CUDA implementation in
``directsht_b200`` can be checked against it.  It is imported only by ``tests/``,
by ``__graft_entry__.smoke()`` and by the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py``; the product path never calls it.

Pinning: every function here is checked in ``tests/test_oracle.py`` against the
golden vectors under ``tests/golden/`` (written by ``tests/golden/make_golden.py``,
which runs the reference's own ``sht.sht.DirectSHT`` on seeded inputs) and against
the reference's published known answers (``sht/test_sht.py:57-59``).

The polar branch of the reference calls ``healpy.rotator.Rotator`` (third party,
no version pinned in ``setup.py:22``, not installed here).  Its point rotation and
``rotate_alm`` are restated below from the mathematics: an active rotation by
+90 degrees about the y axis (ZYZ Euler angles (0, 90, 0)), and the alm rotated back
with Wigner d^l(pi/2) generated by the downward three-term recursion of
Trapani & Navaza (Acta Cryst. A62, 262, 2006).  That restatement is checked against
the exact definition a_lm = sum_i w_i conj(Y_lm(theta_i, phi_i)) computed with
``scipy.special.sph_harm_y``; parity against healpy itself is unpinned.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "x_grid", "healpy_index", "getlm", "plm_table", "dplm_table", "normalize_rows",
    "build_tables", "bin_points", "hermite_weights", "bin_sums", "contract",
    "basic_sht", "rotate_points", "wigner_d_halfpi_column", "rotate_alm_back",
    "direct_sht", "alm2cl", "brute_force_alm", "Tables",
]


# ----------------------------------------------------------------------------
# Grid, indexing
# ----------------------------------------------------------------------------
def x_grid(Nx: int, xmax: float) -> np.ndarray:
    """Uniform spline nodes x_j = j * (xmax/(Nx-1)) (``sht/sht.py:47-48``)."""
    xx = np.arange(Nx, dtype="float64")
    xx *= xmax / float(Nx - 1)
    return xx


def healpy_index(ell, m, Nl: int):
    """Healpy alm index m(2Nl-1-m)/2 + ell (``sht/sht.py:58-67``)."""
    return (m * (2 * Nl - 1 - m)) // 2 + ell


def getlm(Nl: int):
    """(ell, m) of every Healpy index, m-major (``sht/shared_utils.py:76-99``)."""
    ells = np.concatenate([np.arange(m, Nl) for m in range(Nl)])
    ms = np.concatenate([np.full(Nl - m, m) for m in range(Nl)])
    return ells, ms


# ----------------------------------------------------------------------------
# (a) FP64 Ylm / dYlm tables
# ----------------------------------------------------------------------------
def plm_table(Nl: int, xx: np.ndarray) -> np.ndarray:
    """Unnormalised Ylm(x,0) recurrences, rows in Healpy order.

    Follows ``sht/legendre_py.py:4-39`` (m=0 three-term recurrence :18-24, m=ell
    diagonal :28-30, m=ell-1 :32-34) and ``ext_slow_recurrence`` :84-101 for
    ell > m+1, with the same operation order.
    """
    Nx = len(xx)
    sx = np.sqrt(1 - xx ** 2)
    ix = lambda ell, m: (m * (2 * Nl - 1 - m)) // 2 + ell
    P = np.zeros(((Nl * (Nl + 1)) // 2, Nx), dtype="float64")
    P[ix(0, 0), :] = 1.0
    if Nl > 1:
        P[ix(1, 0), :] = xx
    for ell in range(2, Nl):
        i0, i1, i2 = ix(ell, 0), ix(ell - 1, 0), ix(ell - 2, 0)
        P[i0, :] = (2 * ell - 1) * xx * P[i1, :] - (ell - 1) * P[i2, :]
        P[i0, :] /= float(ell)
    for m in range(1, Nl):
        P[ix(m, m), :] = -np.sqrt(1.0 - 1.0 / (2 * m)) * sx * P[ix(m - 1, m - 1), :]
    for m in range(1, Nl - 1):
        P[ix(m + 1, m), :] = np.sqrt(2 * m + 1.0) * xx * P[ix(m, m), :]
    for m in range(0, Nl - 1):
        for ell in range(m + 2, Nl):
            i0, i1, i2 = ix(ell, m), ix(ell - 1, m), ix(ell - 2, m)
            f1 = np.sqrt((ell - m) * 1.0 / (ell + m))
            f2 = np.sqrt((ell - m - 1.0) / (ell + m - 1.0))
            P[i0, :] = (2 * ell - 1) * xx * P[i1, :] - (ell + m - 1) * P[i2, :] * f2
            P[i0, :] *= f1 / (ell - m)
    return P


def dplm_table(Nl: int, xx: np.ndarray, Yv: np.ndarray) -> np.ndarray:
    """d/dx of the unnormalised table (``sht/legendre_py.py:41-60,104-117``)."""
    ix = lambda ell, m: (m * (2 * Nl - 1 - m)) // 2 + ell
    Yd = np.zeros_like(Yv)
    if Nl > 1:
        Yd[ix(1, 0), :] = 1.0
    for ell in range(2, Nl):
        i0, i1 = ix(ell, 0), ix(ell - 1, 0)
        Yd[i0, :] = ell / (1 - xx ** 2) * (Yv[i1, :] - xx * Yv[i0, :])
    omx2 = 1.0 - xx ** 2
    for ell in range(Nl):
        for m in range(1, ell + 1):
            i0, i1 = ix(ell, m), ix(ell - 1, m)
            f = np.sqrt(float(ell - m) / (ell + m))
            Yd[i0, :] = (ell + m) * f * Yv[i1, :] - ell * xx * Yv[i0, :]
            Yd[i0, :] /= omx2
    return Yd


def normalize_rows(Y: np.ndarray, Nl: int) -> np.ndarray:
    """Row scale sqrt((2ell+1)/4pi), in place (``sht/legendre_py.py:67-82``)."""
    for ell in range(Nl):
        f = np.sqrt((2 * ell + 1) / 4.0 / np.pi)
        for m in range(ell + 1):
            Y[healpy_index(ell, m, Nl), :] *= f
    return Y


class Tables:
    """The state ``DirectSHT.__init__`` builds (``sht/sht.py:32-56``)."""

    def __init__(self, Nl: int, Nx: int, xmax: float = 0.75):
        self.Nell, self.Nx, self.xmax = Nl, Nx, xmax
        self.Nlm = Nl * (Nl + 1) // 2
        self.x = x_grid(Nx, xmax)
        Yv = plm_table(Nl, self.x)
        Yd = dplm_table(Nl, self.x, Yv)
        self.Yv = normalize_rows(Yv, Nl)
        self.Yd = normalize_rows(Yd, Nl)


def build_tables(Nl: int, Nx: int, xmax: float = 0.75) -> Tables:
    return Tables(Nl, Nx, xmax)


def table_column(Nl: int, xx: np.ndarray, m: int):
    """Rows l = m..Nl-1 of the normalised Ylm and dYlm tables for one m.

    The same operations as ``plm_table``/``dplm_table``/``normalize_rows`` restricted to
    one column, so large Nl can be checked without the full (Nlm, Nx) tables.
    """
    Nx = len(xx)
    sx = np.sqrt(1 - xx ** 2)
    n = Nl - m
    P = np.zeros((n, Nx))
    pmm = np.ones(Nx)
    for k in range(1, m + 1):
        pmm = -np.sqrt(1.0 - 1.0 / (2 * k)) * sx * pmm
    P[0] = pmm
    if n > 1:
        P[1] = xx.copy() if m == 0 else np.sqrt(2 * m + 1.0) * xx * pmm
    for ell in range(m + 2, Nl):
        f1 = np.sqrt((ell - m) * 1.0 / (ell + m))
        f2 = np.sqrt((ell - m - 1.0) / (ell + m - 1.0))
        P[ell - m] = (2 * ell - 1) * xx * P[ell - m - 1] - (ell + m - 1) * P[ell - m - 2] * f2
        P[ell - m] *= f1 / (ell - m)
    D = np.zeros_like(P)
    omx2 = 1.0 - xx ** 2
    for ell in range(m, Nl):
        i = ell - m
        if m == 0:
            if ell == 1:
                D[i] = 1.0
            elif ell >= 2:
                D[i] = ell / (1 - xx ** 2) * (P[i - 1] - xx * P[i])
        else:
            f = np.sqrt(float(ell - m) / (ell + m))
            prev = P[i - 1] if i >= 1 else 0.0
            D[i] = (ell + m) * f * prev - ell * xx * P[i]
            D[i] /= omx2
    for ell in range(m, Nl):
        f = np.sqrt((2 * ell + 1) / 4.0 / np.pi)
        P[ell - m] *= f
        D[ell - m] *= f
    return P, D


def basic_sht_column(Nl: int, Nx: int, xmax: float, m: int, theta, phi, wt) -> np.ndarray:
    """alm[l, m] for l = m..Nl-1 of ``basic_sht`` (``sht/sht.py:153-283``) for one m,
    from per-m tables (memory O(Nl Nx)) -- the full-size parity check of one column."""
    xx = x_grid(Nx, xmax)
    Yv, Yd = table_column(Nl, xx, m)
    dx = xx[1] - xx[0]
    theta, phi, wt = (np.asarray(a, "float64") for a in (theta, phi, wt))
    x_full = np.cos(theta)
    out = np.zeros(Nl - m, dtype=np.complex128)
    par = (-1.0) ** np.arange(Nl - m)
    for sel, sign in ((x_full >= 0, None), (x_full < 0, par)):
        if not np.any(sel):
            continue
        x = np.abs(x_full[sel])
        j, t = bin_points(x, xx)
        g = hermite_weights(t, wt[sel])
        c, s = np.cos(m * phi[sel]), np.sin(m * phi[sel])
        nb = Nx - 1
        v = np.stack([np.bincount(j, weights=g[k] * c, minlength=nb) - 1j * np.bincount(j, weights=g[k] * s, minlength=nb)
                      for k in range(4)])
        a = Yv[:, :-1] @ v[0] + (dx * Yd[:, :-1]) @ v[1] + Yv[:, 1:] @ v[2] + (dx * Yd[:, 1:]) @ v[3]
        out += a if sign is None else sign * a
    return out


# ----------------------------------------------------------------------------
# (b) bin search + Hermite weights, (c) per-bin sums, (d) contraction
# ----------------------------------------------------------------------------
def bin_points(x: np.ndarray, xx: np.ndarray):
    """Right-open bin index and spline parameter (``sht/sht.py:212-221``).

    Returns (spline_idx, t) for every point, in input order.
    """
    j = np.digitize(x, xx) - 1
    dx = xx[1] - xx[0]
    t = (x - xx[j]) / dx
    return j, t


def hermite_weights(t: np.ndarray, w: np.ndarray) -> np.ndarray:
    """w * {(2t+1)(1-t)^2, t(1-t)^2, t^2(3-2t), t^2(t-1)} (``sht/sht.py:239-240``)."""
    return np.stack([w * ((2 * t + 1) * (1 - t) ** 2), w * (t * (1 - t) ** 2),
                     w * (t ** 2 * (3 - 2 * t)), w * (t ** 2 * (t - 1))])


def bin_sums(Nl: int, j: np.ndarray, phi: np.ndarray, g: np.ndarray):
    """Per-bin v sums for every m (``sht/shared_interp_funcs.py:88-105``,
    ``sht/interp_funcs_py.py:16-35``).

    vr[m,k,b] = sum_{p in bin b} g[k,p] cos(m phi_p), vi likewise with sin.
    Returns (occupied_bins, vr, vi) with vr, vi of shape (Nl, 4, n_occupied).
    """
    order = np.argsort(j, kind="stable")
    js, ph, gs = j[order], phi[order], g[:, order]
    occ, starts = np.unique(js, return_index=True)
    vr = np.zeros((Nl, 4, len(occ)))
    vi = np.zeros((Nl, 4, len(occ)))
    for m in range(Nl):
        c, s = np.cos(m * ph), np.sin(m * ph)
        vr[m] = np.add.reduceat(gs * c, starts, axis=1)
        vi[m] = np.add.reduceat(gs * s, starts, axis=1)
    return occ, vr, vi


def contract(tab: Tables, occ: np.ndarray, vr: np.ndarray, vi: np.ndarray) -> np.ndarray:
    """alm[lm] = sum_b Yv[lm,b] V0 + dx Yd[lm,b] V1 + Yv[lm,b+1] V2 + dx Yd[lm,b+1] V3,
    V = vr - i vi (``sht/sht.py:266-277``, ``sht/interp_funcs_py.py:46-60``).

    Done one m-block of rows at a time instead of materialising the four fancy-indexed
    table copies, so the memory stays at the size of the tables.
    """
    Nl = tab.Nell
    dx = tab.x[1] - tab.x[0]
    vs = vr - 1j * vi
    alm = np.zeros(tab.Nlm, dtype="complex128")
    for m in range(Nl):
        r0 = healpy_index(m, m, Nl)
        r1 = r0 + (Nl - m)
        Yv, Yd = tab.Yv[r0:r1], tab.Yd[r0:r1]
        alm[r0:r1] = (Yv[:, occ] @ vs[m, 0] + (dx * Yd[:, occ]) @ vs[m, 1]
                      + Yv[:, occ + 1] @ vs[m, 2] + (dx * Yd[:, occ + 1]) @ vs[m, 3])
    return alm


def basic_sht(tab: Tables, theta, phi, wt, reg_factor: float = 1.0) -> np.ndarray:
    """Forward transform of points with |cos theta| < xmax (``sht/sht.py:153-283``)."""
    theta, phi, wt = (np.asarray(a, dtype="float64") for a in (theta, phi, wt))
    assert len(theta) == len(phi) and len(phi) == len(wt), \
        "theta,phi,wt must be the same length."
    assert np.all((theta >= 0) & (theta > np.arccos(tab.xmax)) & (theta < np.arccos(-tab.xmax))), \
        "theta must be in [ACos[xmax],ACos[-xmax])."
    Nl = tab.Nell
    w = wt * reg_factor
    ells, ms = getlm(Nl)
    parity = (-1.0) ** (ells - ms)
    x_full = np.cos(theta)
    pos, neg = np.where(x_full >= 0)[0], np.where(x_full < 0)[0]
    if len(pos) == 0 and len(neg) == 0:
        raise ValueError("The theta array seems to be empty!")
    alm = np.zeros(tab.Nlm, dtype="complex128")
    for x, par, idx in ((x_full[pos], 1.0, pos), (np.abs(x_full[neg]), parity, neg)):
        if len(idx) == 0:
            continue
        j, t = bin_points(x, tab.x)
        g = hermite_weights(t, w[idx])
        occ, vr, vi = bin_sums(Nl, j, phi[idx], g)
        alm += par * contract(tab, occ, vr, vi)
    return alm / reg_factor


# ----------------------------------------------------------------------------
# Polar branch: restatement of healpy Rotator((0,90,0), 'ZYZ') and rotate_alm
# ----------------------------------------------------------------------------
_RY90 = np.array([[0.0, 0.0, 1.0], [0.0, 1.0, 0.0], [-1.0, 0.0, 0.0]])


def rotate_points(theta, phi, inverse: bool = False):
    """Rotate points actively by +90 deg about y (or its inverse).

    n = (sin t cos p, sin t sin p, cos t) -> R n with R = Ry(+90) = Rz(0) Ry(90) Rz(0);
    returns (theta', phi') with phi' in [0, 2pi).  Stands in for
    ``hp.rotator.Rotator(rot=(0,90,0), eulertype='ZYZ', deg=True)`` at
    ``sht/sht.py:134-135``.
    """
    theta, phi = np.asarray(theta, "float64"), np.asarray(phi, "float64")
    st = np.sin(theta)
    n = np.stack([st * np.cos(phi), st * np.sin(phi), np.cos(theta)])
    R = _RY90.T if inverse else _RY90
    n2 = R @ n
    t2 = np.arccos(np.clip(n2[2], -1.0, 1.0))
    p2 = np.mod(np.arctan2(n2[1], n2[0]), 2 * np.pi)
    return t2, p2


def _start_column(ell: int):
    """d^ell_{ell,m}(pi/2), m=0..ell, as (mantissa, exponent) pairs.

    Closed form (-1)^(ell-m) 2^-ell sqrt(C(2ell, ell+m)), built from m=ell down with
    the ratio d_{ell,m-1}/d_{ell,m} = -sqrt((ell+m)/(ell-m+1)) so that nothing
    underflows for ell up to a few thousand.
    """
    mant = np.zeros(ell + 1)
    expo = np.zeros(ell + 1, dtype=np.int64)
    v, e = 1.0, -ell
    mant[ell], expo[ell] = v, e
    for m in range(ell, 0, -1):
        v *= -np.sqrt((ell + m) / (ell - m + 1.0))
        f, de = np.frexp(v)
        v, e = f, e + int(de)
        mant[m - 1], expo[m - 1] = v, e
    return mant, expo


def wigner_d_halfpi_column(ell: int) -> np.ndarray:
    """Dense d^ell_{k,m}(pi/2) for k,m in 0..ell (rows k, columns m).

    Downward three-term recursion in the first index for each fixed m
    (Trapani & Navaza 2006):
      sqrt((l+k)(l-k+1)) d_{k-1,m} = 2m d_{k,m} - sqrt((l-k)(l+k+1)) d_{k+1,m},
    started from the closed-form d_{ell,m}; values are carried with a per-column
    binary exponent while they are below the double range.
    """
    mant, expo = _start_column(ell)
    D = np.zeros((ell + 1, ell + 1))
    m = np.arange(ell + 1, dtype="float64")
    cur = mant.copy()
    nxt = np.zeros(ell + 1)
    E = expo.astype(np.int64).copy()
    scale = np.where(E > -1000, np.ldexp(1.0, np.maximum(E, -1000)), 0.0)
    D[ell] = cur * scale
    for k in range(ell, 0, -1):
        c1 = np.sqrt((ell - k) * (ell + k + 1.0))
        c2 = 1.0 / np.sqrt((ell + k) * (ell - k + 1.0))
        prv = (2.0 * m * cur - c1 * nxt) * c2
        big = np.abs(prv) > 2.0 ** 256
        prv[big] *= 2.0 ** -256
        cur[big] *= 2.0 ** -256
        E[big] += 256
        scale = np.where(E > -1000, np.ldexp(1.0, np.maximum(E, -1000)), 0.0)
        nxt, cur = cur, prv
        D[k - 1] = cur * scale
    return D


def rotate_alm_back(alm_rot: np.ndarray, Nl: int) -> np.ndarray:
    """alm of the original points from alm of the points rotated by ``rotate_points``.

    a_lm = sum_{m'=-l..l} d^l_{m'm}(pi/2) a'_lm'.  With a'_{l,-m'} = (-1)^m' conj(a'_lm')
    this is Re a_lm = d_{0m} a'_l0 + 2 sum_{m'>0, l+m+m' even} d_{m'm} Re a'_lm' and
    Im a_lm = 2 sum_{m'>0, l+m+m' odd} d_{m'm} Im a'_lm'.  Stands in for
    ``Rotator(rot=(0,90,0), eulertype='ZYZ', deg=True, inv=True).rotate_alm`` at
    ``sht/sht.py:138-139``.
    """
    out = np.zeros_like(alm_rot)
    for ell in range(Nl):
        idx = healpy_index(ell, np.arange(ell + 1), Nl)
        a = alm_rot[idx]
        D = wigner_d_halfpi_column(ell)                     # D[k, m] = d_{k,m}
        k = np.arange(ell + 1)[:, None]
        m = np.arange(ell + 1)[None, :]
        even = ((ell + m + k) % 2 == 0)
        wk = np.where(k == 0, 1.0, 2.0)
        re = np.sum(np.where(even, D * wk * a.real[:, None], 0.0), axis=0)
        im = np.sum(np.where(~even & (k > 0), 2.0 * D * a.imag[:, None], 0.0), axis=0)
        out[idx] = re + 1j * im
    return out


class AlmRotator:
    """``rotate_alm_back`` with the d^l(pi/2) matrices computed once (the CPU baseline's
    stand-in for healpy's ``rotate_alm`` inside its timed region).

    For each l the sums of ``rotate_alm_back`` split by the parities of k and m: with
    p = l % 2, Re a_lm takes k = m + p (mod 2) and Im a_lm the other k, so each l is four
    dense matrix-vector products over strided views of one stored matrix."""

    def __init__(self, Nl: int):
        self.Nl = Nl
        self.D = [wigner_d_halfpi_column(ell) for ell in range(Nl)]

    def __call__(self, alm_rot: np.ndarray) -> np.ndarray:
        Nl = self.Nl
        out = np.zeros_like(alm_rot)
        for ell in range(Nl):
            idx = healpy_index(ell, np.arange(ell + 1), Nl)
            a = alm_rot[idx]
            D = self.D[ell]
            wre = a.real.copy()
            wre[1:] *= 2.0
            wim = 2.0 * a.imag
            wim[0] = 0.0
            re = np.empty(ell + 1)
            im = np.empty(ell + 1)
            p = ell % 2
            for mp in (0, 1):              # parity of m
                ke = (mp + p) % 2          # k parity of the real part (l + m + k even)
                ko = 1 - ke
                re[mp::2] = wre[ke::2] @ D[ke::2, mp::2]
                im[mp::2] = wim[ko::2] @ D[ko::2, mp::2]
            out[idx] = re + 1j * im
        return out


def direct_sht(tab: Tables, t, p, w) -> np.ndarray:
    """``DirectSHT.__call__`` (``sht/sht.py:112-150``): polar/equatorial split,
    rotation of the polar points, transform, rotation of their alm back."""
    t, p, w = (np.asarray(a, dtype="float64") for a in (t, p, w))
    alms = np.zeros(tab.Nlm, dtype="complex128")
    xval = np.abs(np.cos(t))
    pol = np.nonzero(xval >= tab.xmax)[0]
    equ = np.nonzero(xval < tab.xmax)[0]
    ok = True
    if len(pol) > 0:
        ok = False
        tp, pp = rotate_points(t[pol], p[pol])
        try:
            rlms = basic_sht(tab, tp, pp, w[pol])
            alms += rotate_alm_back(rlms, tab.Nell)
            ok = True
        except AssertionError:
            pass
    if ok and len(equ) > 0:
        alms += basic_sht(tab, t[equ], p[equ], w[equ])
    return alms


def alm2cl(alm: np.ndarray, Nl: int) -> np.ndarray:
    """1/(2l+1) sum_m |a_lm|^2 with m>0 counted twice (``sht/sht.py:95-109``)."""
    cl = np.zeros(Nl)
    for ell in range(Nl):
        cl[ell] = alm[healpy_index(ell, 0, Nl)].real ** 2
        for m in range(1, ell + 1):
            a = alm[healpy_index(ell, m, Nl)]
            cl[ell] += 2 * (a.real ** 2 + a.imag ** 2)
        cl[ell] /= 2 * ell + 1.0
    return cl


def brute_force_alm(theta, phi, w, Nl: int) -> np.ndarray:
    """Exact a_lm = sum_i w_i conj(Y_lm(theta_i, phi_i)) with scipy (small cases only)."""
    from scipy.special import sph_harm_y
    alm = np.zeros(Nl * (Nl + 1) // 2, dtype="complex128")
    for m in range(Nl):
        for ell in range(m, Nl):
            alm[healpy_index(ell, m, Nl)] = np.sum(w * np.conj(sph_harm_y(ell, m, theta, phi)))
    return alm


# ----------------------------------------------------------------------------
# Mode coupling of pseudo-Cl (next to the transform: MaskDeconvolution)
# ----------------------------------------------------------------------------
def threej000(l1: int, l2: int, l3: int, _cache={}) -> float:
    """Wigner 3j (l1 l2 l3; 0 0 0) by the reference's recursion (``sht/threej000.py:9-41``):
    sort j1 >= j2 >= j3; zero for odd J; (-1)^j1/sqrt(2 j1 + 1) at j3 = 0, j1 = j2; else
    sqrt((J-2j2-1)(J-2j3+2) / ((J-2j2)(J-2j3+1))) times the value at (j1, j2+1, j3-1)."""
    J = l1 + l2 + l3
    j1 = max(l1, l2, l3)
    j3 = min(l1, l2, l3)
    j2 = J - j1 - j3
    key = (j1, j2, j3)
    if key in _cache:
        return _cache[key]
    if J % 2:
        res = 0.0
    elif j3 == 0:
        res = (-1.0) ** j1 / np.sqrt(2 * j1 + 1.0) if j1 == j2 else 0.0
    else:
        num = (J - 2 * j2 - 1) * (J - 2 * j3 + 2)
        den = (J - 2 * j2) * (J - 2 * j3 + 1)
        res = np.sqrt(float(num) / float(den)) * threej000(j1, j2 + 1, j3 - 1)
    _cache[key] = res
    return res


def mode_coupling(Nl: int, W_l: np.ndarray) -> np.ndarray:
    """M[l1, l2] = (2 l2 + 1)/(4 pi) sum_l3 (2 l3 + 1) W[l3] (l1 l2 l3; 000)^2 for l1, l2 < Nl,
    W right-padded with zeros to 2 Nl - 1 (``sht/mask_deconvolution.py:28-32, 171-192``).
    Pure Python loops: small Nl only."""
    W = np.pad(np.asarray(W_l, "float64"), (0, max(0, 2 * Nl - 1 - len(W_l))))
    M = np.zeros((Nl, Nl))
    for l1 in range(Nl):
        for l2 in range(Nl):
            s = 0.0
            for l3 in range(abs(l1 - l2), l1 + l2 + 1):
                if (l1 + l2 + l3) % 2 == 0:
                    s += (2 * l3 + 1) * W[l3] * threej000(l1, l2, l3) ** 2
            M[l1, l2] = s * (2 * l2 + 1)
    return M / (4 * np.pi)


def mode_coupling_closed_form(Nl: int, W_l: np.ndarray) -> np.ndarray:
    """The same matrix from the closed form of (l1 l2 l3; 000)^2 with log-gamma (vectorised
    over l3): an independent check for sizes where the recursion above is too slow."""
    from scipy.special import gammaln
    W = np.pad(np.asarray(W_l, "float64"), (0, max(0, 2 * Nl - 1 - len(W_l))))
    M = np.zeros((Nl, Nl))
    for l1 in range(Nl):
        for l2 in range(Nl):
            l3 = np.arange(abs(l1 - l2), l1 + l2 + 1, 2)
            J = l1 + l2 + l3
            g = J // 2
            lw = (gammaln(J - 2 * l1 + 1) + gammaln(J - 2 * l2 + 1) + gammaln(J - 2 * l3 + 1) - gammaln(J + 2)
                  + 2 * (gammaln(g + 1) - gammaln(g - l1 + 1) - gammaln(g - l2 + 1) - gammaln(g - l3 + 1)))
            Wl3 = np.where(l3 < len(W), W[np.minimum(l3, len(W) - 1)], 0.0)
            M[l1, l2] = np.sum((2 * l3 + 1) * Wl3 * np.exp(lw)) * (2 * l2 + 1)
    return M / (4 * np.pi)
