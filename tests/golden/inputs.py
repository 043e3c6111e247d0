"""Seeded point sets for the golden vectors (shared by make_golden.py and the tests).

Each case is regenerated from its seed with ``numpy.random.default_rng`` (PCG64), so
only the reference's outputs are stored.  ``entry`` says which reference entry point
produced the fixture: ``call`` = ``DirectSHT.__call__`` (polar rotation included),
``basic`` = ``DirectSHT.basic_sht`` (|cos theta| < xmax only).
"""
from __future__ import annotations

import numpy as np

CASES = {
    # Full sky, Nl=256, Nx=512, N=1e5, w=1, seed 0 (the CPU-runnable reference case).
    "c1_full_sky": dict(Nl=256, Nx=512, N=100_000, seed=0, kind="full", wkind="ones", entry="call"),
    "small_call": dict(Nl=48, Nx=96, N=3000, seed=1, kind="full", wkind="uniform", entry="call"),
    "small_basic_mixed_sign": dict(Nl=32, Nx=64, N=2000, seed=2, kind="band", lo=-0.74, hi=0.74,
                                   wkind="lognormal", entry="basic"),
    "basic_pos_only": dict(Nl=40, Nx=80, N=1500, seed=3, kind="band", lo=0.05, hi=0.7,
                           wkind="uniform", entry="basic"),
    "basic_neg_only": dict(Nl=40, Nx=80, N=1500, seed=4, kind="band", lo=-0.7, hi=-0.05,
                           wkind="uniform", entry="basic"),
    "nodes_exact": dict(Nl=24, Nx=48, N=600, seed=5, kind="nodes", wkind="uniform", entry="basic"),
    "one_bin": dict(Nl=32, Nx=64, N=800, seed=6, kind="band", lo=0.3, hi=0.305,
                    wkind="uniform", entry="basic"),
    "cap_c2like": dict(Nl=64, Nx=128, N=20000, seed=7, kind="c2", wkind="lognormal", entry="call"),
    "reg_factor": dict(Nl=20, Nx=40, N=500, seed=8, kind="band", lo=-0.6, hi=0.6, wkind="uniform",
                       entry="basic", reg=1000.0),
    "single_point": dict(Nl=16, Nx=32, N=1, seed=9, kind="band", lo=-0.5, hi=0.5, wkind="uniform",
                         entry="basic"),
    "xmax_0p8": dict(Nl=30, Nx=60, N=2500, seed=10, kind="full", wkind="uniform", entry="call",
                     xmax=0.8),
    "test_alm_example": dict(Nl=40, Nx=1024, N=1000, seed=0, kind="test_alm", wkind="ones",
                             entry="call"),
}


def x_nodes(Nx: int, xmax: float) -> np.ndarray:
    xx = np.arange(Nx, dtype="float64")
    xx *= xmax / float(Nx - 1)
    return xx


def make_inputs(name: str):
    """(theta, phi, w) float64 arrays for a named case."""
    s = CASES[name]
    rng = np.random.default_rng(s["seed"])
    N = s["N"]
    kind = s["kind"]
    if kind == "full":
        cost = rng.uniform(-1.0, 1.0, N)
        phi = rng.uniform(0.0, 2 * np.pi, N)
    elif kind == "band":
        cost = rng.uniform(s["lo"], s["hi"], N)
        phi = rng.uniform(0.0, 2 * np.pi, N)
    elif kind == "c2":
        cost = rng.uniform(np.cos(1.2), np.cos(0.3), N)
        phi = rng.uniform(0.0, 1.5 * np.pi, N)
    elif kind == "nodes":
        xx = x_nodes(s["Nx"], s.get("xmax", 0.75))
        j = rng.integers(0, s["Nx"] - 1, N)
        sign = np.where(rng.uniform(size=N) < 0.5, -1.0, 1.0)
        cost = sign * xx[j]
        phi = rng.uniform(0.0, 2 * np.pi, N)
    elif kind == "test_alm":
        # The point set of the reference's csht/test_alm.py:68-70.
        cost = np.concatenate([np.linspace(-0.7, -0.3, 500), np.linspace(0.2, 0.8, 500)])
        phi = np.linspace(0.0, 2 * np.pi, 1000)
    else:
        raise ValueError(kind)
    theta = np.arccos(cost)
    wk = s["wkind"]
    if wk == "ones":
        w = np.ones(N)
    elif wk == "uniform":
        w = rng.uniform(0.5, 1.5, N)
    elif wk == "lognormal":
        w = rng.lognormal(0.0, 0.5, N)
    else:
        raise ValueError(wk)
    return theta, phi, w
