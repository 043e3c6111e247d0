#!/usr/bin/env python
"""Writes the golden vectors under tests/golden/ by running the reference itself.

Imports the reference's numpy/numba path (``sht.sht.DirectSHT``; JAX absent) from the
reference checkout, with the test-only healpy stand-in in ``_healpy_shim`` on the path
for its polar branch, and saves inputs and outputs as compressed .npz files.  Inputs
are regenerated from their seeds by ``tests/golden/inputs.py`` so that the fixtures
stay small.  Needs the reference checkout; the fixtures it writes are committed.

    python tests/golden/make_golden.py --ref <reference checkout>   (or DSHT_REFERENCE=<checkout>)
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(HERE, "_healpy_shim"))
sys.path.insert(0, HERE)

import inputs as I  # noqa: E402


def _quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DSHT_REFERENCE"),
                    help="the reference checkout (default: $DSHT_REFERENCE)")
    ap.add_argument("--skip-c1", action="store_true")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or DSHT_REFERENCE")
    sys.path.insert(0, args.ref)
    with contextlib.redirect_stdout(io.StringIO()):
        from sht.sht import DirectSHT  # noqa: E402

    # 1. Tables: the rows and x indices that sht/test_sht.py:31-66 inspects.
    t0 = time.time()
    sht = _quiet(DirectSHT, 500, 1024)
    ix = np.array([0, 1024 // 3, 2 * 1024 // 3, 1023])
    rows = [(ell, m) for ell in range(45) for m in range(ell + 1)]
    rows += [(ell, m) for ell in (100, 250, 499) for m in (0, 1, 50, 99, ell - 1, ell) if m <= ell]
    rows = sorted(set(rows))
    yv = np.array([sht.get_Ylm(l, m)[ix] for l, m in rows])
    yd = np.array([sht.get_dYlm(l, m)[ix] for l, m in rows])
    full = [(2, 0), (10, 10), (37, 5), (499, 3)]
    yv_full = np.array([sht.get_Ylm(l, m) for l, m in full])
    yd_full = np.array([sht.get_dYlm(l, m) for l, m in full])
    np.savez_compressed(os.path.join(HERE, "tables_nl500_nx1024.npz"), Nl=500, Nx=1024, xmax=0.75,
                        x=sht.x, ix=ix, rows=np.array(rows), yv=yv, yd=yd,
                        full_rows=np.array(full), yv_full=yv_full, yd_full=yd_full)
    print(f"tables: {time.time() - t0:.1f}s")

    # 2. Transforms through DirectSHT.__call__ / basic_sht on seeded point sets.
    cases = dict(I.CASES)
    if args.skip_c1:
        cases.pop("c1_full_sky")
    for name, spec in cases.items():
        t0 = time.time()
        theta, phi, w = I.make_inputs(name)
        d = _quiet(DirectSHT, spec["Nl"], spec["Nx"], xmax=spec.get("xmax", 0.75))
        if spec["entry"] == "call":
            alm = _quiet(d, theta, phi, w.copy())
        else:
            alm = _quiet(d.basic_sht, theta, phi, w.copy(), reg_factor=spec.get("reg", 1.0))
        cl = d.alm2cl(alm)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), alm=alm, cl=cl,
                            Nl=spec["Nl"], Nx=spec["Nx"], xmax=spec.get("xmax", 0.75))
        print(f"{name}: N={len(theta)} {time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
