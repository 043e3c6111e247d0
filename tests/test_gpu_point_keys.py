"""The sort key of every point, index for index, against the oracle's binning.

The count pass decides most keys from FP32 sines and cosines and hands the points near a
decision boundary (bin edges, the polar cut, the sign of x, the rotated range) to the FP64
path.  This checks that the split is invisible: random points and points placed on every
kind of boundary, from 1e-12 to 1e-5 away, get the key the reference's binning gives --
the set of sht/sht.py:128-130 and :193, the bin numpy.digitize(|x|, x_grid) - 1 of
sht/sht.py:212 -- and the same flags.  Points within 1e-13 of a boundary, where the host's
and the device's correctly-rounded-to-an-ulp sines may disagree, are left out."""
import numpy as np
import pytest
import torch

from directsht_b200 import DirectSHT
from directsht_b200 import _lib as L
from oracle import dsht_oracle as O

pytestmark = pytest.mark.gpu

DROP = 0xFFFFFFFF
F_THETA, F_POLAR, F_HAS_POLAR = 1, 2, 4
AMBIG = 1e-13


def _expected(th, ph, Nx, xmax, mode):
    """Keys, flags and the ambiguous mask from the reference's rules (FP64, numpy)."""
    nb = Nx - 1
    xx = O.x_grid(Nx, xmax)
    dx = xx[1] - xx[0]
    c, st = np.cos(th), np.sin(th)
    keys = np.full(th.shape, DROP, np.int64)
    amb = np.zeros(th.shape, bool)
    flags = 0
    in_theta = (th >= 0.0) & (th > np.arccos(xmax)) & (th < np.arccos(-xmax))
    if mode == L.DSHT_MODE_CALL:
        pol = np.abs(c) >= xmax
        equ = np.abs(c) < xmax
        amb |= np.abs(np.abs(c) - xmax) < AMBIG
        z = -(st * np.cos(ph))
        x = np.where(pol, z, c)
        inside = np.where(pol, (z < xmax) & (z > -xmax), in_theta)
        amb |= pol & (np.abs(np.abs(z) - xmax) < AMBIG)
        if np.any(pol):
            flags |= F_HAS_POLAR
        if np.any(pol & ~inside):
            flags |= F_POLAR
        if np.any(equ & ~inside):
            flags |= F_THETA
        setb = np.where(pol, 2, 0)
        live = (pol | equ) & inside
    else:
        x = c
        inside = in_theta
        if np.any(~inside):
            flags |= F_THETA
        setb = np.zeros(th.shape, np.int64)
        live = inside
    setb = setb + (~(x >= 0.0))
    ax = np.abs(x)
    j = np.digitize(ax, xx) - 1
    ok = live & (j >= 0) & (j < nb)
    keys[ok] = (setb * nb + j)[ok]
    edge = np.rint(ax / dx) * dx
    amb |= (np.abs(ax - edge) < AMBIG) | (ax < AMBIG)
    return keys, flags, amb


def _device_keys(d, th, ph, mode):
    t = torch.from_numpy(th).cuda()
    p = torch.from_numpy(ph).cuda()
    keys = torch.empty(len(th), dtype=torch.int32, device="cuda")
    flags = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.check(d._lib.dsht_test_point_keys(d._plan, t.data_ptr(), p.data_ptr(), len(th), mode, keys.data_ptr(),
                                        flags.data_ptr(), None))
    return keys.cpu().numpy().view(np.uint32).astype(np.int64), int(flags.cpu().numpy().view(np.uint32)[0])


def _boundary_points(rng, Nx, xmax, n):
    """theta, phi on and beside every decision boundary of the binning."""
    dx = xmax / (Nx - 1)
    offs = np.array([1e-12, 1e-10, 1e-9, 1e-8, 1e-7, 5e-7, 1e-6, 2e-6, 3e-6, 5e-6, 1e-5])
    d = rng.choice(np.concatenate([offs, -offs]), n)
    sgn = rng.choice([-1.0, 1.0], n)
    th, ph = [], []
    # bin edges of equatorial points, both hemispheres
    e = rng.integers(1, Nx - 1, n) * dx
    th.append(np.arccos(np.clip(sgn * (e + d), -1, 1)))
    ph.append(rng.uniform(0, 2 * np.pi, n))
    # the polar cut |cos theta| = xmax, and the equator
    th.append(np.arccos(np.clip(sgn * (xmax + d), -1, 1)))
    ph.append(rng.uniform(0, 2 * np.pi, n))
    th.append(np.arccos(d))
    ph.append(rng.uniform(0, 2 * np.pi, n))
    # polar points whose rotated x = -sin(theta) cos(phi) sits on a bin edge, on 0, or on the
    # rotated range's end
    tp = rng.uniform(0.02, np.arccos(xmax) * 0.999, n)
    tp = np.where(rng.random(n) < 0.5, tp, np.pi - tp)
    smax = np.sin(tp)
    kmax = np.floor(smax / dx).astype(np.int64)
    target = np.where(rng.random(n) < 0.8, rng.integers(0, np.maximum(kmax, 1)) * dx + d, d)
    target = np.where(rng.random(n) < 0.1, xmax + d, target) * sgn
    cp = np.clip(-target / smax, -1, 1)
    th.append(tp)
    ph.append(np.arccos(cp) * rng.choice([-1.0, 1.0], n) % (2 * np.pi))
    return np.concatenate(th), np.concatenate(ph)


@pytest.mark.parametrize("Nx", [64, 2048, 8192, 12288])
def test_keys_random_and_boundary_points(Nx):
    rng = np.random.default_rng(Nx)
    xmax = 0.95
    d = DirectSHT(16, Nx, xmax)
    N = 400_000
    th = np.arccos(rng.uniform(-1, 1, N))
    ph = rng.uniform(0, 2 * np.pi, N)
    tb, pb = _boundary_points(rng, Nx, xmax, 100_000)
    th, ph = np.concatenate([th, tb]), np.concatenate([ph, pb])
    for mode in (L.DSHT_MODE_CALL,):
        got, gflags = _device_keys(d, th, ph, mode)
        want, wflags, amb = _expected(th, ph, Nx, xmax, mode)
        bad = (got != want) & ~amb
        assert not bad.any(), (Nx, np.nonzero(bad)[0][:5], got[bad][:5], want[bad][:5])
        assert amb.mean() < 1e-3
        assert gflags == wflags


def test_keys_basic_mode_and_odd_angles():
    """basic_sht mode (equatorial band only, out-of-band theta flagged), NaN theta, theta
    outside [0, pi] and phi far outside [0, 2 pi): the FP64 path decides those."""
    rng = np.random.default_rng(7)
    Nx, xmax = 512, 0.9
    d = DirectSHT(16, Nx, xmax)
    n = 50_000
    band = rng.uniform(np.arccos(xmax), np.arccos(-xmax), n)
    got, gflags = _device_keys(d, band, rng.uniform(0, 2 * np.pi, n), L.DSHT_MODE_BASIC)
    want, wflags, amb = _expected(band, np.zeros(n), Nx, xmax, L.DSHT_MODE_BASIC)
    assert not ((got != want) & ~amb).any() and gflags == wflags == 0
    th = np.concatenate([band[:1000], [0.01, 3.13, -0.3, 3.5, np.nan]])
    got, gflags = _device_keys(d, th, np.zeros(len(th)), L.DSHT_MODE_BASIC)
    want, wflags, amb = _expected(th, np.zeros(len(th)), Nx, xmax, L.DSHT_MODE_BASIC)
    assert not ((got != want) & ~amb).any() and gflags == wflags == F_THETA
    # __call__ with odd angles: polar points of huge phi, theta < 0 and > pi, NaN
    th = np.concatenate([np.arccos(rng.uniform(-1, 1, 5000)), [0.05, 0.05, -0.4, -2.0, 4.0, 7.0, np.nan]])
    ph = np.concatenate([rng.uniform(-50, 50, 5000), [1e3, -1e4, 0.3, 1.0, 2.0, 0.5, 0.0]])
    got, gflags = _device_keys(d, th, ph, L.DSHT_MODE_CALL)
    want, wflags, amb = _expected(th, ph, Nx, xmax, L.DSHT_MODE_CALL)
    assert not ((got != want) & ~amb).any()
    assert gflags == wflags
