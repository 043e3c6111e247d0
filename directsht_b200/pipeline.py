"""Back-to-back transforms of host-resident point sets with the copies overlapped.

The reference transforms one point set per ``DirectSHT.__call__`` (``sht/sht.py:112-150``)
and every call starts from host arrays.  ``Pipeline`` runs such a sequence on the GPU so
that the host->device copy of transform i+1 and the device->host copy of transform i-1
overlap the kernels of transform i: inputs are staged in pinned host buffers, copied on
a copy stream, transformed on a compute stream with ``dsht_enqueue_maps`` (no host
synchronisation), and the alm come back to pinned host memory.  ``depth`` transforms may
be in flight; each slot owns its device buffers and workspace.
"""
from __future__ import annotations

import ctypes as ct
from collections import deque

import numpy as np
import torch

from . import _lib as L


class _Slot:
    def __init__(self, d, N, nmaps, w_dtype, device):
        self.N, self.nmaps = N, nmaps
        self.h = [torch.empty(N, dtype=torch.float64).pin_memory(), torch.empty(N, dtype=torch.float64).pin_memory(),
                  torch.empty((nmaps, N), dtype=w_dtype).pin_memory()]
        self.dv = [torch.empty_like(x, device=device) for x in self.h]
        nb = ct.c_size_t()
        L.check(d._lib.dsht_workspace_size_maps(d._plan, N, nmaps, ct.byref(nb)))
        self.ws = torch.empty(max(int(nb.value), 1), dtype=torch.uint8, device=device)
        self.alm = torch.empty((nmaps, d.Nlm), dtype=torch.complex128, device=device)
        self.out = torch.empty((nmaps, d.Nlm), dtype=torch.complex128).pin_memory()
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.status_h = torch.zeros(1, dtype=torch.int32).pin_memory()
        self.done = torch.cuda.Event()
        self.copied = torch.cuda.Event()
        self.busy = False
        self.ticket = None


class Ticket:
    """Handle of one submitted transform; keeps its result once the slot is reused."""

    def __init__(self, slot):
        self.slot = slot
        self.value = None
        self.error = None


class Pipeline:
    """Overlapped transforms of host point sets on one plan (``DirectSHT``).

    ``submit(theta, phi, w)`` copies the host arrays into a free slot's pinned buffers,
    enqueues copy-in, transform and copy-out, and returns a ticket; ``result(ticket)``
    waits for that transform and returns its complex128 alm (numpy, shape (Nlm,) for one
    map or (nmaps, Nlm)).  Sizes up to ``max_N`` points and ``nmaps`` maps per call.
    """

    def __init__(self, sht, max_N: int, nmaps: int = 1, w_dtype=np.float64, depth: int = 2):
        self.d = sht
        self.device = sht.device
        self.max_N, self.nmaps = int(max_N), int(nmaps)
        self.w_dtype = np.dtype(w_dtype)
        tdt = torch.float32 if self.w_dtype == np.float32 else torch.float64
        with torch.cuda.device(self.device):
            self.slots = [_Slot(sht, self.max_N, self.nmaps, tdt, self.device) for _ in range(max(depth, 1))]
            self.copy_stream = torch.cuda.Stream(device=self.device)
            self.compute_stream = torch.cuda.Stream(device=self.device)
        self.inflight: deque = deque()
        self.next_slot = 0
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    def submit(self, theta, phi, w):
        """Queue one transform.  theta, phi: N float64 values; w: N or (nmaps, N) weights.
        numpy arrays are first copied into the slot's pinned buffers; pinned CPU tensors
        (float64 theta/phi, weights of the pipeline's dtype, contiguous) are copied to the
        device directly and must stay unchanged until the transform's result is taken."""
        N = len(theta)
        pinned = all(isinstance(a, torch.Tensor) and a.is_pinned() for a in (theta, phi, w))
        if pinned:
            wt = w if w.dim() == 2 else w[None, :]
            src = [theta, phi, wt]
            wshape = tuple(wt.shape)
        else:
            w = np.asarray(w)
            if w.ndim == 1:
                w = w[None, :]
            wshape = w.shape
        if N > self.max_N or wshape != (self.nmaps, N) or len(phi) != N:
            raise ValueError(f"pipeline sized for N <= {self.max_N}, {self.nmaps} maps; got N={N}, w {wshape}")
        s = self.slots[self.next_slot]
        if s.busy:  # the slot's transform must finish (its result is kept in its ticket)
            self._collect(s.ticket)
        self.next_slot = (self.next_slot + 1) % len(self.slots)
        if not pinned:
            s.h[0][:N].numpy()[:] = theta
            s.h[1][:N].numpy()[:] = phi
            s.h[2][:, :N].numpy()[:] = w.astype(self.w_dtype, copy=False)
            src = [s.h[0][:N], s.h[1][:N], s.h[2][:, :N]]
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(s.done)  # the slot's previous transform has finished
            s.dv[0][:N].copy_(src[0], non_blocking=True)
            s.dv[1][:N].copy_(src[1], non_blocking=True)
            s.dv[2][:, :N].copy_(src[2], non_blocking=True)
            s.copied.record(self.copy_stream)
        self.h2d_bytes = 16 * N + self.w_dtype.itemsize * self.nmaps * N
        cs = self.compute_stream
        cs.wait_event(s.copied)
        wd = s.dv[2]
        L.check(self.d._lib.dsht_enqueue_maps(
            self.d._plan, L.ptr(s.dv[0]), L.ptr(s.dv[1]), L.ptr(wd),
            L.DSHT_W_F32 if self.w_dtype == np.float32 else L.DSHT_W_F64, N, self.nmaps, wd.stride(0),
            L.DSHT_MODE_CALL, L.ptr(s.alm), L.ptr(s.status), L.ptr(s.ws), s.ws.numel(), ct.c_void_p(cs.cuda_stream)))
        with torch.cuda.stream(cs):
            s.out.copy_(s.alm, non_blocking=True)
            s.status_h.copy_(s.status, non_blocking=True)
            s.done.record(cs)
        self.d2h_bytes = s.out.numel() * 16
        s.busy = True
        t = Ticket(s)
        s.ticket = t
        self.inflight.append(t)
        return t

    def _collect(self, t):
        """Wait for the ticket's transform and keep its result (or error) in the ticket."""
        if t.slot is None:
            return
        s = t.slot
        s.done.synchronize()
        if t in self.inflight:
            self.inflight.remove(t)
        s.busy = False
        t.slot = None
        rc = self.d._lib.dsht_status(int(s.status_h[0]) & 0xffffffff, L.DSHT_MODE_CALL)
        out = s.out.numpy().copy()
        if rc == L.DSHT_ERR_POLAR_RANGE:
            out[:] = 0  # DirectSHT.__call__ returns zeros (sht/sht.py:141-148)
        elif rc == L.DSHT_ERR_THETA_RANGE:
            t.error = AssertionError("theta must be in [ACos[xmax],ACos[-xmax]).")
        elif rc != L.DSHT_OK:
            t.error = L.DSHTError(rc, L.last_error())
        t.value = out[0] if self.nmaps == 1 else out

    def result(self, ticket):
        """The alm of a submitted transform (waits for it)."""
        self._collect(ticket)
        if ticket.error is not None:
            raise ticket.error
        return ticket.value

    def drain(self):
        return [self.result(t) for t in list(self.inflight)]
