"""Uneven batches of transforms: many point sets of different sizes and different (Nl, Nx).

The reference transforms one point set per ``DirectSHT.__call__`` (``sht/sht.py:112-150``)
and has no batch layer; this module is the B200 batch runner around the library's
``dsht_enqueue_batch``:

* one plan per (Nl, Nx, xmax) stays resident (``PlanCache``); plans whose FP64 tables would
  not fit keep the compact 4-byte fixed-point tables only;
* the transforms of one plan are dealt into sub-batches (largest first, balanced by points)
  that run on their own CUDA streams; inside a sub-batch the library's tensor-core
  contraction shares one read of the tables between up to eight transforms, and one
  rotation recursion serves them all;
* the whole batch is enqueued without any host synchronisation, so it can be captured once
  into a CUDA graph and replayed with a single launch (``TransformBatch.capture``);
* ``autotune`` picks, per plan, the piece size of the bin sums, the maps per contraction
  pass and the number of sub-batch streams by timing the candidates on the batch itself,
  and keeps the choice in a JSON cache keyed by device, plan and size profile.
"""
from __future__ import annotations

import ctypes as ct
import itertools
import json
import math
import os
import threading

import numpy as np
import torch

from . import _lib as L
from .sht import DirectSHT


def table_bytes(Nl: int, Nx: int, compact: bool, mixed: bool = False) -> int:
    """Device bytes of a plan's tables: the FP64 pair (16 B per entry pair) unless compact,
    plus the 4-byte fixed-point digit tables (4 planes of 2 Nx bytes per row, rounded up to
    64) when the plan is compact or runs at the mixed level."""
    nlm = Nl * (Nl + 1) // 2
    digits = 4 * nlm * ((2 * Nx + 63) // 64 * 64)
    if compact:
        return digits
    return 2 * nlm * Nx * 8 + (digits if mixed else 0)


class PlanCache:
    """Resident plans keyed by (Nl, Nx, xmax) on one device.

    ``compact_min_nl``: plans with Nl at or above it keep the compact (4-byte fixed-point)
    tables only (at Nl=2048, Nx=4096 the FP64 pair alone is 137 GB, the compact tables 69 GB).
    Plans are built on first use and kept.
    """

    def __init__(self, device=None, precision="mixed", compact_min_nl=2048):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else torch.device(device).index or 0)
        self.precision = precision
        self.compact_min_nl = compact_min_nl
        self._plans: dict = {}
        self._lock = threading.Lock()

    def get(self, Nl: int, Nx: int, xmax: float = 0.75) -> DirectSHT:
        key = (int(Nl), int(Nx), float(xmax))
        with self._lock:
            d = self._plans.get(key)
            if d is None:
                compact = self.precision == "mixed" and Nl >= self.compact_min_nl and Nx <= 8192
                d = DirectSHT(Nl, Nx, xmax, device=self.device, precision=self.precision, compact_tables=compact)
                self._plans[key] = d
            return d

    def resident_bytes(self) -> int:
        return sum(table_bytes(d.Nell, d.Nx, d._f32_only, d.precision == "mixed") for d in self._plans.values())

    def plans(self):
        return dict(self._plans)


class _SubBatch:
    """Transforms of one plan enqueued by one dsht_enqueue_batch call on one stream."""

    def __init__(self, plan: DirectSHT, idx, thetas, phis, ws_, Ns, alms, status, device):
        self.plan, self.idx = plan, list(idx)
        n = len(self.idx)
        self.n = n
        vp = lambda xs: (ct.c_void_p * n)(*[x.data_ptr() for x in xs])
        self.th = vp([thetas[i] for i in self.idx])
        self.ph = vp([phis[i] for i in self.idx])
        self.w = vp([ws_[i] for i in self.idx])
        self.alm = vp([alms[i] for i in self.idx])
        self.N = (ct.c_int64 * n)(*[Ns[i] for i in self.idx])
        self.status = status
        nb = ct.c_size_t()
        L.check(plan._lib.dsht_workspace_size_batch(plan._plan, max(max(self.N), 1), n, ct.byref(nb)))
        self.ws = torch.empty(max(int(nb.value), 1), dtype=torch.uint8, device=device)
        self.stream = torch.cuda.Stream(device=device)

    def enqueue(self, mode):
        L.check(self.plan._lib.dsht_enqueue_batch(self.plan._plan, self.n, self.th, self.ph, self.w, self.N, mode,
                                                  self.alm, L.ptr(self.status), L.ptr(self.ws), self.ws.numel(),
                                                  ct.c_void_p(self.stream.cuda_stream)))


def _deal(idx, Ns, k):
    """Split transform indices into k groups of similar point totals (largest first)."""
    bins = [[] for _ in range(k)]
    load = [0] * k
    for i in sorted(idx, key=lambda i: -Ns[i]):
        j = int(np.argmin(load))
        bins[j].append(i)
        load[j] += max(Ns[i], 1)
    return [b for b in bins if b]


class TransformBatch:
    """A fixed set of transforms ``(Nl, Nx, theta, phi, w)`` (CUDA float64 tensors; numpy
    arrays are copied to the device once) run together.  ``alms[i]`` receives transform i
    (complex128, Healpy order, DirectSHT.__call__ semantics)."""

    def __init__(self, cache: PlanCache, transforms, mode="call", config=None):
        self.cache = cache
        self.device = cache.device
        self.mode = L.DSHT_MODE_CALL if mode == "call" else L.DSHT_MODE_BASIC
        dev = self.device
        as_dev = lambda a: (a.to(device=dev, dtype=torch.float64).contiguous() if isinstance(a, torch.Tensor)
                            else torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev))
        self.keys, self.thetas, self.phis, self.ws_, self.Ns = [], [], [], [], []
        for t in transforms:
            Nl, Nx, th, ph, w = t[:5]
            xmax = t[5] if len(t) > 5 else 0.75
            self.keys.append((int(Nl), int(Nx), float(xmax)))
            self.thetas.append(as_dev(th))
            self.phis.append(as_dev(ph))
            self.ws_.append(as_dev(w))
            self.Ns.append(int(len(th)))
        self.n = len(self.keys)
        self.status = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.alms = [torch.zeros(cache.get(*k).Nlm, dtype=torch.complex128, device=dev) for k in self.keys]
        self.groups = {}
        for i, k in enumerate(self.keys):
            self.groups.setdefault(k, []).append(i)
        self.config = dict(config or {})
        self.graph = None
        self._build()

    # -- layout ---------------------------------------------------------------------
    def _build(self):
        self.subs = []
        for key, idx in self.groups.items():
            plan = self.cache.get(*key)
            cfg = self.config.get(key, {})
            plan.tune(piece_max=cfg.get("piece_max", 0), maps_per_pass=cfg.get("maps_per_pass", 0))
            for part in _deal(idx, self.Ns, int(cfg.get("streams", 1))):
                # status words of the part: a contiguous view is not possible for an arbitrary
                # index set, so each part writes its own small tensor, gathered in check().
                st = torch.zeros(len(part), dtype=torch.int32, device=self.device)
                self.subs.append((_SubBatch(plan, part, self.thetas, self.phis, self.ws_, self.Ns, self.alms, st,
                                            self.device), key, cfg))
        self.graph = None

    def points_ell(self) -> int:
        """Sum of N x Nl over the transforms (the unit of the throughput metric)."""
        return int(sum(n * k[0] for n, k in zip(self.Ns, self.keys)))

    # -- execution ------------------------------------------------------------------
    def _enqueue_all(self, main):
        for sb, key, cfg in self.subs:
            plan = sb.plan
            plan.tune(piece_max=cfg.get("piece_max", 0), maps_per_pass=cfg.get("maps_per_pass", 0))
            sb.stream.wait_stream(main)
            sb.enqueue(self.mode)
            main.wait_stream(sb.stream)

    def run(self):
        """Enqueue every transform on its sub-batch stream (no synchronisation)."""
        if self.graph is not None:
            self.graph.replay()
            return
        self._enqueue_all(torch.cuda.current_stream(self.device))

    def capture(self):
        """Capture the whole batch into one CUDA graph (after one eager run, which sets the
        kernels' attributes and warms the plans); later ``run`` calls replay it."""
        self.run()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream(device=self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.graph(g, stream=side):
            self._enqueue_all(side)
        torch.cuda.current_stream(self.device).wait_stream(side)
        self.graph = g
        return g

    def release(self):
        self.graph = None

    def check(self):
        """After the work has finished: raise for the first transform that failed; a
        transform whose polar points could not be rotated into range gets zero alm, as
        DirectSHT.__call__ returns."""
        lib = L.load()
        for sb, _, _ in self.subs:
            flags = sb.status.cpu().numpy().astype(np.uint32)
            for j, f in enumerate(flags):
                rc = lib.dsht_status(int(f), self.mode)
                i = sb.idx[j]
                if rc == L.DSHT_ERR_POLAR_RANGE and self.mode == L.DSHT_MODE_CALL:
                    self.alms[i].zero_()
                elif rc == L.DSHT_ERR_THETA_RANGE:
                    raise AssertionError(f"transform {i}: theta must be in [ACos[xmax],ACos[-xmax]).")
                else:
                    L.check(rc)


# ---------------------------------------------------------------------------------------
def _profile_key(batch: TransformBatch, key) -> str:
    idx = batch.groups[key]
    Ns = np.array([batch.Ns[i] for i in idx], dtype=np.float64)
    # size profile: count and the log2 buckets of N (the choice depends on both)
    buckets = np.bincount(np.clip(np.log2(np.maximum(Ns, 1)).astype(int) // 2, 0, 15), minlength=16)
    return f"{key[0]}x{key[1]}x{key[2]}|n={len(idx)}|" + ",".join(str(int(b)) for b in buckets)


def default_cache_path() -> str:
    base = os.environ.get("DSHT_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "directsht_b200",
                                                              "autotune.json")
    return base


def autotune(batch: TransformBatch, path: str | None = None, reps: int = 2, verbose=False) -> dict:
    """Choose per plan (piece_max, maps_per_pass, streams) by timing each candidate on the
    batch's own transforms with CUDA events; reuse earlier choices from the JSON cache at
    ``path`` for the same device, plan and size profile.  Returns the configuration, which
    is also installed in ``batch``."""
    path = path or default_cache_path()
    dev_name = torch.cuda.get_device_name(batch.device)
    try:
        with open(path) as f:
            store = json.load(f)
    except (OSError, ValueError):
        store = {}
    config = {}
    main = torch.cuda.current_stream(batch.device)
    for key in batch.groups:
        pk = f"{dev_name}|{batch.cache.precision}|nufft|{_profile_key(batch, key)}"
        if pk in store:
            config[key] = store[pk]["config"]
            continue
        plan = batch.cache.get(*key)
        f32 = plan.precision == "mixed"
        n = len(batch.groups[key])
        # the NUFFT bin sums of mixed plans pay one FFT per piece: larger pieces
        pieces = [0, 4096, 16384] if f32 else [0, 512, 1024, 2048]
        per_pass = [0, 4] if f32 else [0]  # mixed plans: 8 (0) or 4 transforms per table read
        streams = [s for s in (1, 2, 4) if s <= n]
        best = None
        for pm, mp, ns in itertools.product(pieces, per_pass, streams):
            cfg = {"piece_max": pm, "maps_per_pass": mp, "streams": ns}
            sub = TransformBatch.__new__(TransformBatch)
            sub.__dict__.update(batch.__dict__)
            sub.groups = {key: batch.groups[key]}
            sub.config = {key: cfg}
            sub.graph = None
            sub._build()
            sub.run()
            torch.cuda.synchronize(batch.device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(main)
            for _ in range(reps):
                sub.run()
            e1.record(main)
            torch.cuda.synchronize(batch.device)
            ms = e0.elapsed_time(e1) / reps
            if verbose:
                print(f"autotune {key} {cfg}: {ms:.3f} ms", flush=True)
            if best is None or ms < best[0]:
                best = (ms, cfg)
            del sub
        config[key] = best[1]
        store[pk] = {"config": best[1], "ms": best[0]}
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as f:
            json.dump(store, f, indent=1, sort_keys=True)
    except OSError:
        pass
    batch.config = config
    batch._build()
    return config
