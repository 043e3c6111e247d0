#!/usr/bin/env python
"""Writes tests/golden/mode_coupling.npz by running the reference's own MaskDeconvolution
(``sht/mask_deconvolution.py``, with its Wigner 3j table ``sht/threej000.py``) on a seeded
window: the mode-coupling matrix, a linear and a sqrt binning, the window matrices and the
decoupled / normalised bandpowers of a seeded pseudo-Cl.  Needs the reference checkout.

    python tests/golden/make_golden_coupling.py --ref <reference checkout>   (or DSHT_REFERENCE=<checkout>)
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DSHT_REFERENCE"),
                    help="the reference checkout (default: $DSHT_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or DSHT_REFERENCE")
    sys.path.insert(0, args.ref)
    with contextlib.redirect_stdout(io.StringIO()):
        from sht.mask_deconvolution import MaskDeconvolution
    rng = np.random.default_rng(21)
    Nl = 64
    # a smooth, positive window with structure up to 2 lmax (as a sky mask's)
    ell = np.arange(2 * Nl - 1)
    W = np.exp(-ell / 9.0) * (1.0 + 0.3 * np.cos(ell / 3.0)) + rng.uniform(0, 1e-3, ell.size)
    Cl = 1.0 / (ell[:Nl] + 10.0) + rng.uniform(0, 1e-3, Nl)
    with contextlib.redirect_stdout(io.StringIO()):
        md = MaskDeconvolution(Nl, W.copy(), verbose=False)
        b_lin = md.binning_matrix("linear", start=2, step=8)
        b_sqrt = md.binning_matrix("sqrt", start=2, step=4)
        ells_d, Cb_d = md(Cl, b_lin, mode="deconvolution")
        ells_n, Cb_n = md(Cl, b_lin, mode="normalization")
        win_d = md.window_matrix(b_sqrt, mode="deconvolution")
        win_n = md.window_matrix(b_sqrt, mode="normalization")
        Mdebug = md.get_M(debug=True)
    np.savez_compressed(os.path.join(HERE, "mode_coupling.npz"), Nl=Nl, W=W, Cl=Cl, Mll=md.Mll, Mdebug=Mdebug,
                        b_lin=b_lin, b_sqrt=b_sqrt, ells_d=ells_d, Cb_d=Cb_d, ells_n=ells_n, Cb_n=Cb_n,
                        win_d=win_d, win_n=win_n)
    print("mode_coupling.npz written")


if __name__ == "__main__":
    main()
