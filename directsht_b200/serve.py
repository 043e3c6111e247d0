"""Request loop for a stream of transform requests with continuous batching.

The reference has no serving layer (one ``DirectSHT.__call__`` per point set,
``sht/sht.py:112-150``).  This module keeps the Ylm/dYlm tables resident per (Nl, Nx)
(``batch.PlanCache``), admits requests by their device-memory footprint, and runs every
admitted request on its own slot (a CUDA stream with its own workspace), so requests that
arrive while others run are admitted as soon as a slot and memory are free and their work
overlaps on the device.  Each request's alm come back to pinned host memory; the latency
of a request is submit -> alm on the host.

The policy (``Admission``) is plain Python and is tested on the CPU with a fake
executor; ``GpuExecutor`` enqueues a request with ``dsht_enqueue_maps`` (no host
synchronisation) and reports completion through a CUDA event.
"""
from __future__ import annotations

import collections
import ctypes as ct
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L


@dataclass
class Request:
    """One transform request: ``nmaps`` weight maps on one point set (numpy arrays)."""
    Nl: int
    Nx: int
    theta: np.ndarray
    phi: np.ndarray
    w: np.ndarray            # (nmaps, N) float32/float64, or (N,)
    xmax: float = 0.75
    rid: int = 0
    t_submit: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    future: Future = field(default_factory=Future)

    @property
    def N(self) -> int:
        return int(len(self.theta))

    @property
    def nmaps(self) -> int:
        return 1 if np.ndim(self.w) == 1 else int(np.shape(self.w)[0])

    @property
    def key(self):
        return (int(self.Nl), int(self.Nx), float(self.xmax))

    def points_ell(self) -> int:
        return self.N * self.nmaps * int(self.Nl)


class Admission:
    """Arrival-order admission under a slot limit and a device-memory budget.

    A request is admitted when a slot is free and its footprint fits in what the budget
    has left.  The head of the queue is never overtaken by more than ``max_bypass`` later
    requests (small requests may pass a large one that waits for memory, but not forever).
    A request larger than the whole budget is rejected.
    """

    def __init__(self, budget_bytes: int, slots: int, max_bypass: int = 8):
        self.budget = int(budget_bytes)
        self.slots = int(slots)
        self.max_bypass = int(max_bypass)
        self.used = 0
        self.running = 0
        self.queue: collections.deque = collections.deque()
        self._bypassed = 0

    def push(self, req, footprint: int):
        self.queue.append((req, int(footprint)))

    def pop_admissible(self):
        """Requests to start now, in order, with their footprints; and rejected ones."""
        start, rejected = [], []
        i = 0
        while self.queue and i < len(self.queue) and self.running < self.slots:
            req, fp = self.queue[i]
            if fp > self.budget:
                del self.queue[i]
                rejected.append(req)
                continue
            if self.used + fp <= self.budget:
                del self.queue[i]
                self.used += fp
                self.running += 1
                start.append((req, fp))
                if i > 0:
                    self._bypassed += 1
                    if self._bypassed >= self.max_bypass:
                        break  # the head waits; nothing else may pass it now
                else:
                    self._bypassed = 0
                continue
            if i == 0 and self._bypassed >= self.max_bypass:
                break  # the head waits; nothing else may pass it now
            i += 1
        return start, rejected

    def release(self, footprint: int):
        self.used -= int(footprint)
        self.running -= 1


class GpuExecutor:
    """Runs a request on a slot stream: pinned H2D copies, ``dsht_enqueue_maps``, alm D2H to
    pinned memory, completion event."""

    def __init__(self, cache):
        import torch
        self.torch = torch
        self.cache = cache
        self.device = cache.device

    def footprint(self, req: Request) -> int:
        d = self.cache.get(*req.key)
        nb = ct.c_size_t()
        L.check(d._lib.dsht_workspace_size_maps(d._plan, req.N, req.nmaps, ct.byref(nb)))
        wbytes = np.asarray(req.w).dtype.itemsize * req.N * req.nmaps
        return int(nb.value) + 16 * req.N + wbytes + 16 * d.Nlm * req.nmaps + 4096

    def prepare(self, req: Request):
        """Stage the request's arrays in pinned host memory (on the submitting thread)."""
        torch = self.torch
        w = np.asarray(req.w)
        if w.ndim == 1:
            w = w[None, :]
        if w.dtype not in (np.float32, np.float64):
            w = w.astype(np.float64)
        req._pinned = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                       for a in (np.asarray(req.theta, np.float64), np.asarray(req.phi, np.float64), w)]

    def start(self, req: Request):
        torch = self.torch
        d = self.cache.get(*req.key)
        stream = torch.cuda.Stream(device=self.device)
        if getattr(req, "_pinned", None) is None:
            self.prepare(req)
        h = req._pinned
        w = h[2].numpy()
        with torch.cuda.stream(stream):
            dv = [x.to(self.device, non_blocking=True) for x in h]
            nb = ct.c_size_t()
            L.check(d._lib.dsht_workspace_size_maps(d._plan, req.N, req.nmaps, ct.byref(nb)))
            ws = torch.empty(max(int(nb.value), 1), dtype=torch.uint8, device=self.device)
            alm = torch.empty((req.nmaps, d.Nlm), dtype=torch.complex128, device=self.device)
            status = torch.zeros(1, dtype=torch.int32, device=self.device)
            rc = d._lib.dsht_enqueue_maps(d._plan, L.ptr(dv[0]), L.ptr(dv[1]), L.ptr(dv[2]),
                                          L.DSHT_W_F32 if w.dtype == np.float32 else L.DSHT_W_F64, req.N,
                                          req.nmaps, req.N, L.DSHT_MODE_CALL, L.ptr(alm), L.ptr(status), L.ptr(ws),
                                          ws.numel(), ct.c_void_p(stream.cuda_stream))
            L.check(rc)
            out = torch.empty((req.nmaps, d.Nlm), dtype=torch.complex128).pin_memory()
            out.copy_(alm, non_blocking=True)
            st_h = torch.empty(1, dtype=torch.int32).pin_memory()
            st_h.copy_(status, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        # the tensors stay referenced until completion (the caching allocator is stream-aware)
        req._pinned = None
        return {"event": ev, "keep": (h, dv, ws, alm, status), "out": out, "status": st_h, "stream": stream}

    def done(self, handle) -> bool:
        return handle["event"].query()

    def result(self, req: Request, handle):
        lib = L.load()
        rc = lib.dsht_status(int(handle["status"][0]) & 0xffffffff, L.DSHT_MODE_CALL)
        out = handle["out"].numpy()
        if rc == L.DSHT_ERR_POLAR_RANGE:
            out = out * 0  # DirectSHT.__call__ returns zeros (sht/sht.py:141-148)
        elif rc != L.DSHT_OK:
            raise L.DSHTError(rc, "request failed")
        return out


class Server:
    """Continuous-batching request loop on one device.

    ``submit`` returns a Future for the (nmaps, Nlm) complex128 alm.  One scheduler thread
    admits queued requests (``Admission``), starts them on the executor, and polls the
    running ones; a finished request frees its slot and memory at once.
    """

    def __init__(self, executor, budget_bytes: int, slots: int = 8, poll_s: float = 2e-4, max_bypass: int = 8):
        self.ex = executor
        self.adm = Admission(budget_bytes, slots, max_bypass)
        self.poll_s = poll_s
        self.running = []
        self.finished = []
        self.rejected = []
        self._lock = threading.Lock()
        self._cv = threading.Condition(self._lock)
        self._stop = False
        self._thread = threading.Thread(target=self._loop, name="dsht-serve", daemon=True)
        self._next_id = 0
        self.max_running = 0

    def start(self):
        self._thread.start()
        return self

    def submit(self, req: Request) -> Future:
        fp = self.ex.footprint(req)
        prep = getattr(self.ex, "prepare", None)
        if prep is not None:
            prep(req)
        with self._cv:
            req.rid = self._next_id
            self._next_id += 1
            req.t_submit = time.perf_counter()
            self.adm.push(req, fp)
            self._cv.notify()
        return req.future

    def stop(self, drain=True, timeout=None):
        t0 = time.perf_counter()
        if drain:
            while True:
                with self._lock:  # adm.running counts admitted requests until their release
                    if not self.adm.queue and self.adm.running == 0:
                        break
                if timeout is not None and time.perf_counter() - t0 > timeout:
                    break
                time.sleep(1e-3)
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join()

    def _loop(self):
        while True:
            with self._cv:
                if self._stop:
                    return
                if not self.adm.queue and self.adm.running == 0:
                    self._cv.wait(timeout=0.05)
                    continue
                start, rejected = self.adm.pop_admissible()
            for req in rejected:
                req.future.set_exception(MemoryError(f"request {req.rid} needs more than the memory budget"))
                self.rejected.append(req)
            for req, fp in start:
                req.t_admit = time.perf_counter()
                try:
                    h = self.ex.start(req)
                except Exception as exc:  # reported to the caller, slot freed
                    with self._lock:
                        self.adm.release(fp)
                    req.future.set_exception(exc)
                    continue
                self.running.append((req, fp, h))
            self.max_running = max(self.max_running, len(self.running))
            still = []
            for req, fp, h in self.running:
                if self.ex.done(h):
                    req.t_done = time.perf_counter()
                    try:
                        req.future.set_result(self.ex.result(req, h))
                    except Exception as exc:
                        req.future.set_exception(exc)
                    with self._lock:
                        self.adm.release(fp)
                    self.finished.append(req)
                else:
                    still.append((req, fp, h))
            with self._lock:
                self.running = still
            if not start:
                time.sleep(self.poll_s)

    def stats(self) -> dict:
        lat = np.array([r.t_done - r.t_submit for r in self.finished]) * 1e3
        wait = np.array([r.t_admit - r.t_submit for r in self.finished]) * 1e3
        if len(lat) == 0:
            return {"requests": 0}
        t0 = min(r.t_submit for r in self.finished)
        t1 = max(r.t_done for r in self.finished)
        pe = sum(r.points_ell() for r in self.finished)
        return {"requests": len(lat), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean()), "queue_p50_ms": float(np.percentile(wait, 50)),
                "makespan_s": t1 - t0, "points_ell": int(pe), "points_ell_per_s": pe / max(t1 - t0, 1e-9),
                "max_concurrent": int(self.max_running), "rejected": len(self.rejected)}


# ---------------------------------------------------------------------------------------
def cap_points(rng, N, alpha, return_centre=False):
    """N points uniform in a spherical cap of half-angle alpha around a random centre:
    cos of the distance ~ U[cos alpha, 1], azimuth ~ U[0, 2 pi), rotated to the centre.
    Returns (theta, phi) [and the centre (theta0, phi0)]."""
    cd = rng.uniform(np.cos(alpha), 1.0, N)
    az = rng.uniform(0.0, 2 * np.pi, N)
    sd = np.sqrt(np.maximum(0.0, 1.0 - cd * cd))
    v = np.stack([sd * np.cos(az), sd * np.sin(az), cd])          # around +z
    th0 = np.arccos(rng.uniform(-1.0, 1.0))   # random centre
    ph0 = rng.uniform(0, 2 * np.pi)
    # rotation taking +z to (th0, ph0): R = Rz(ph0) Ry(th0)
    c, s = np.cos(th0), np.sin(th0)
    x = c * v[0] + s * v[2]
    z = -s * v[0] + c * v[2]
    y = v[1]
    cp, sp = np.cos(ph0), np.sin(ph0)
    x, y = cp * x - sp * y, sp * x + cp * y
    theta = np.arccos(np.clip(z, -1.0, 1.0))
    phi = np.mod(np.arctan2(y, x), 2 * np.pi)
    if return_centre:
        return theta, phi, (th0, ph0)
    return theta, phi


def poisson_requests(rng, n, rate_hz, Nls=(256, 512, 1024, 2048), n_range=(1e4, 3e7), maps=(1, 16),
                     alpha_range=(0.2, np.pi)):
    """n requests of the serving workload with Poisson arrival offsets (seconds)."""
    out = []
    t = 0.0
    for i in range(n):
        t += rng.exponential(1.0 / rate_hz)
        Nl = int(rng.choice(Nls))
        N = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        k = int(rng.integers(maps[0], maps[1] + 1))
        th, ph = cap_points(rng, N, rng.uniform(*alpha_range))
        w = rng.uniform(0.5, 1.5, (k, N)).astype(np.float32)
        out.append((t, Request(Nl, 2 * Nl, th, ph, w)))
    return out


def replay(server: Server, timed_requests, time_scale: float = 1.0):
    """Submit the requests at their arrival offsets (wall clock); returns the futures."""
    t0 = time.perf_counter()
    futs = []
    for t, req in timed_requests:
        delay = t * time_scale - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        futs.append(server.submit(req))
    return futs
