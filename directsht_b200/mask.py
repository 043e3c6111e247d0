"""Mode-decoupling of pseudo-Cl with the mode-coupling matrix built on the GPU.

Mirrors the reference's ``MaskDeconvolution`` (``sht/mask_deconvolution.py:14-243``): the
same constructor arguments, ``__call__`` (MASTER deconvolution or the shot-noise
normalisation of Baleato Lizancos & White 2023), ``window_matrix``,
``convolve_theory_Cls``, ``binning_matrix``, ``get_Mbb_inv``, ``decouple_Cls`` and ``W``.
The O(lmax^3) part, ``get_M``, runs in the library's ``mode_coupling_kernel``
(``dsht_mode_coupling``), which forms every Wigner 3j (l1 l2 l3; 0 0 0) it needs on the fly
instead of tabulating all (2 Nl)^3 / 6 of them (``sht/threej000.py``); the binned matrices
are Nbin x Nbin and stay in numpy on the host, as in the reference.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from . import _lib as L


def mode_coupling_matrix(Nl: int, W_l, device=None) -> np.ndarray:
    """M[l1, l2] for l1, l2 < Nl from the window W_l (``sht/mask_deconvolution.py:171-192``),
    computed on the GPU; W_l is used up to index 2 Nl - 2 (missing entries are zero)."""
    lib = L.load()
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index or 0)
    W = torch.as_tensor(np.ascontiguousarray(np.asarray(W_l, dtype=np.float64)[: 2 * Nl - 1]), device=dev)
    M = torch.empty((Nl, Nl), dtype=torch.float64, device=dev)
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        L.check(lib.dsht_mode_coupling(int(Nl), L.ptr(W), int(W.numel()), L.ptr(M), ct.c_void_p(stream)))
    return M.cpu().numpy()


class MaskDeconvolution:
    """Mode-coupling of pseudo-Cls (``sht/mask_deconvolution.py:14``)."""

    def __init__(self, Nl, W_l, verbose=True, precompute_3j_and_Mll=True, device=None):
        """:param Nl: number of multipoles; lmax = Nl - 1.
        :param W_l: window function at every ell, right-padded with zeros to 2 lmax + 1.
        :param verbose: print progress, as the reference does.
        :param precompute_3j_and_Mll: build the mode-coupling matrix now (else on first use).
            No 3j table is kept: the kernel forms the symbols it needs."""
        self.Nl = Nl
        self.lmax = Nl - 1
        pad = max(0, 2 * Nl - 1 - W_l.size)
        self.W_l = np.pad(W_l, (0, pad), "constant", constant_values=0)
        self.device = device
        if precompute_3j_and_Mll:
            if verbose:
                print("Computing the mode-coupling matrix...")
            self.Mll = self.get_M()
        else:
            self.Mll = None

    def __call__(self, Cl, bins, mode="deconvolution"):
        """(binned ells, mode-decoupled or normalised bandpowers) of the pseudo-Cl
        (``sht/mask_deconvolution.py:53-95``)."""
        if len(Cl) < self.Nl:
            Clx = np.pad(Cl, (0, self.Nl - len(Cl)), "constant", constant_values=0)
        elif len(Cl) > self.Nl:
            Clx = Cl[: self.Nl]
        else:
            Clx = Cl
        Cb = np.dot(bins, Clx)
        binned_ells = np.dot(bins, np.arange(self.Nl)) / np.sum(bins, axis=1)
        if mode == "deconvolution":
            return binned_ells, self.decouple_Cls(self.get_Mbb_inv(bins), Cb)
        if mode == "normalization":
            return binned_ells, self.compute_normalization_factor() * Cb
        raise RuntimeError("Unknown mode. Must be 'deconvolution' or 'normalization'.")

    def compute_normalization_factor(self):
        """1 / (sum_l (2l+1) W_l / 4pi), which leaves shot noise unchanged
        (``sht/mask_deconvolution.py:97-104``)."""
        ells = np.arange(len(self.W_l))
        return 1.0 / (np.sum(self.W_l * (2 * ells + 1)) / (4 * np.pi))

    def convolve_theory_Cls(self, Clt, bins, mode="deconvolution"):
        """(binned ells, window matrix . Clt) (``sht/mask_deconvolution.py:106-123``)."""
        assert len(Clt) >= self.Nl, "Clt must be provided up to lmax"
        binned_ells = np.dot(bins, np.arange(self.Nl)) / np.sum(bins, axis=1)
        return binned_ells, np.dot(self.window_matrix(bins, mode), Clt[: self.Nl])

    def window_matrix(self, bins, mode="deconvolution"):
        """Matrix taking a theory Cl to the binned, decoupled pseudo-spectrum
        (``sht/mask_deconvolution.py:125-153``)."""
        if self.Mll is None:
            self.Mll = self.get_M()
        if mode == "deconvolution":
            return np.dot(self.get_Mbb_inv(bins), np.dot(bins, self.Mll))
        if mode == "normalization":
            return self.compute_normalization_factor() * np.dot(bins, self.Mll)
        raise RuntimeError("Unknown mode. Must be 'deconvolution' or 'normalization'.")

    def W(self, l, debug=False):
        """Window at multipole l; debug=True gives the full-sky window (4 pi at l = 0)
        (``sht/mask_deconvolution.py:155-169``)."""
        if debug:
            return 4 * np.pi if l == 0 else 0
        return self.W_l[l]

    def get_M(self, debug=False):
        """The (lmax+1) x (lmax+1) mode-coupling matrix on the GPU; debug=True uses the
        full-sky window, for which it is the identity (``sht/mask_deconvolution.py:171-192``)."""
        W = self.W_l if not debug else np.concatenate([[4 * np.pi], np.zeros(2 * self.Nl - 2)])
        return mode_coupling_matrix(self.Nl, W, self.device)

    def get_Mbb_inv(self, bins):
        """Inverse of the binned mode-coupling matrix (``sht/mask_deconvolution.py:194-210``)."""
        if self.Mll is None:
            self.Mll = self.get_M()
        bins_no_wt = np.zeros_like(bins)
        bins_no_wt[bins > 0] = 1.0
        Mbb = np.dot(np.dot(bins, self.Mll), bins_no_wt.T)
        return np.linalg.inv(Mbb)

    def binning_matrix(self, type="linear", start=0, step=16):
        """Binning matrix B with B . vec the binned vec (``sht/mask_deconvolution.py:212-238``)."""
        Nl = self.lmax + 1
        bins = np.zeros((Nl, Nl))
        if type == "linear":
            dell = lambda ell: step
        elif type == "sqrt":
            dell = lambda ell: int(np.ceil(np.sqrt(4.0 * ell) + step))
        else:
            raise RuntimeError("Unknown step type.")
        ii = 0
        l0 = start
        l1 = l0 + dell(l0)
        while l1 <= Nl:
            bins[ii, l0:min(l1, Nl)] = 1 / float(l1 - l0)
            l0, l1 = l1, l1 + dell(l1)
            ii += 1
        return bins[:ii, :]

    def decouple_Cls(self, Minv, Cb):
        """Mode-decoupled bandpowers Minv . Cb (``sht/mask_deconvolution.py:240-246``)."""
        return np.dot(Minv, Cb)
