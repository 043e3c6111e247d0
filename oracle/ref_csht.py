"""ctypes driver for the reference's own C/OpenMP transform -- TEST AND BASELINE ONLY.

Loads ``oracle/_ref/sht_helper.so`` (built by ``oracle/Makefile`` from the reference's
``csht/sht_helper.c``) and drives it the way the reference's ``csht/sht.py:78-140``
does: points split by the sign of cos(theta), each half sorted by |cos(theta)|,
``do_transform`` called per half, alm = carr - i*sarr, the parity (-1)^(l-m) applied
to the cos(theta) < 0 half.  The polar/equatorial split of ``csht/calc_alms.py:11-27``
is added on top, with the oracle's rotation restatement standing in for healpy.

Used as a cross-check in the tests and as the CPU baseline of ``bench.py``.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import dsht_oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "sht_helper.so")

_dp = ct.POINTER(ct.c_double)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _lib():
    lib = ct.CDLL(LIB_PATH)
    lib.make_table.argtypes = [ct.c_int, ct.c_int, ct.c_double, _dp, _dp]
    lib.make_table.restype = ct.c_int
    lib.do_transform.argtypes = [ct.c_int, ct.c_int, ct.c_double, _dp, _dp, ct.c_int,
                                 _dp, _dp, _dp, _dp, _dp]
    lib.do_transform.restype = ct.c_int
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class RefCSHT:
    """Tables from ``make_table`` (``csht/sht_helper.c:18-116``) kept in host RAM."""

    def __init__(self, Nl: int, Nx: int, xmax: float = 0.75):
        self.lib = _lib()
        self.Nell, self.Nx, self.xmax = Nl, Nx, xmax
        self.Nlm = Nl * (Nl + 1) // 2
        self.Yv = np.zeros(self.Nlm * Nx)
        self.Yd = np.zeros(self.Nlm * Nx)
        rc = self.lib.make_table(Nl, Nx, xmax, _p(self.Yv), _p(self.Yd))
        if rc != 0:
            raise MemoryError("make_table failed")
        ells, ms = O.getlm(Nl)
        self.parity = (-1.0) ** (ells - ms)

    def basic(self, theta, phi, wt) -> np.ndarray:
        """Equatorial transform as ``csht/sht.py:78-140`` does it."""
        cost = np.cos(np.asarray(theta, "float64"))
        phi = np.asarray(phi, "float64")
        wt = np.asarray(wt, "float64")
        alm = np.zeros(self.Nlm, dtype=np.complex128)
        carr = np.zeros(self.Nlm)
        sarr = np.zeros(self.Nlm)
        for sel, key, par in ((np.nonzero(cost < 0)[0], lambda c: -c, self.parity),
                              (np.nonzero(cost >= 0)[0], lambda c: c, 1.0)):
            if len(sel) == 0:
                continue
            ii = sel[np.argsort(key(cost[sel]))]
            tt = np.ascontiguousarray(cost[ii])
            pp = np.ascontiguousarray(phi[ii])
            ww = np.ascontiguousarray(wt[ii])
            rc = self.lib.do_transform(self.Nell, self.Nx, self.xmax, _p(self.Yv), _p(self.Yd),
                                       len(ii), _p(tt), _p(pp), _p(ww), _p(carr), _p(sarr))
            if rc != 0:
                raise MemoryError("do_transform failed")
            alm += par * (carr - 1j * sarr)
        return alm

    def __call__(self, t, p, w) -> np.ndarray:
        """Polar/equatorial split of ``csht/calc_alms.py:11-27``."""
        t, p, w = (np.asarray(a, "float64") for a in (t, p, w))
        alms = np.zeros(self.Nlm, dtype=np.complex128)
        xval = np.abs(np.cos(t))
        pol = np.nonzero(xval >= self.xmax)[0]
        equ = np.nonzero(xval < self.xmax)[0]
        if len(pol) > 0:
            tp, pp = O.rotate_points(t[pol], p[pol])
            alms += O.rotate_alm_back(self.basic(tp, pp, w[pol]), self.Nell)
        if len(equ) > 0:
            alms += self.basic(t[equ], p[equ], w[equ])
        return alms
