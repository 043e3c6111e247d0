"""GPU test of dsht_execute_noalloc, the transform entry point that allocates nothing.

Callers that cannot allocate device memory (their framework owns the GPU's memory pool,
their plugin host forbids allocations, or their loop cannot absorb the synchronisation a
cudaMalloc implies) use this entry point; its scratch is a fixed 64 MiB device array
inside the library.  The test calls it twice in a row through the C ABI and checks each
result against dsht_execute, which allocates a workspace as usual.  Collected last so a
run that stops at the first failure has already run everything else; it also passes on
its own in a fresh process.
"""
import ctypes as ct

import numpy as np
import pytest
import torch

from directsht_b200 import DirectSHT
from directsht_b200 import _lib as L

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_MIXED = 1e-7


def _points(N, seed):
    rng = np.random.default_rng(seed)
    th = torch.from_numpy(np.arccos(rng.uniform(-1, 1, N))).cuda()
    ph = torch.from_numpy(rng.uniform(0, 2 * np.pi, N)).cuda()
    w = torch.from_numpy(rng.uniform(0.5, 1.5, N)).cuda()
    return th, ph, w


def _with_workspace(lib, d, th, ph, w):
    alm = torch.empty(d.Nlm, dtype=torch.complex128, device="cuda")
    nbytes = ct.c_size_t()
    L.check(lib.dsht_workspace_size(d._plan, th.numel(), ct.byref(nbytes)))
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device="cuda")
    s = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    L.check(lib.dsht_execute(d._plan, L.ptr(th), L.ptr(ph), L.ptr(w), th.numel(), L.DSHT_MODE_CALL, L.ptr(alm),
                             L.ptr(ws), ws.numel(), s))
    return alm.cpu().numpy()


def _no_alloc(lib, d, th, ph, w):
    alm = torch.empty(d.Nlm, dtype=torch.complex128, device="cuda")
    s = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    L.check(lib.dsht_execute_noalloc(d._plan, L.ptr(th), L.ptr(ph), L.ptr(w), th.numel(), L.DSHT_MODE_CALL,
                                     L.ptr(alm), s))
    return alm.cpu().numpy()


def test_no_alloc_matches_execute_on_two_calls_in_a_row():
    lib = L.load()
    assert lib.dsht_noalloc_scratch_bytes() == 64 << 20
    d = DirectSHT(256, 512)  # Nl=256, Nx=512, N=1e5 fits the fixed scratch
    for seed, N in ((0, 100_000), (1, 37_000)):  # two calls, different sizes, back to back
        th, ph, w = _points(N, seed)
        ref = _with_workspace(lib, d, th, ph, w)
        got = _no_alloc(lib, d, th, ph, w)
        assert np.abs(got - ref).max() <= TOL_FP64 * np.abs(ref).max()


def test_no_alloc_mixed_precision_two_calls():
    """The tensor-core level keeps FP32 partial sums and piece maxima in the same fixed
    array; its results equal dsht_execute's on the same plan within the mixed tolerance."""
    lib = L.load()
    d = DirectSHT(256, 512, precision="mixed")
    for seed, N in ((3, 100_000), (4, 52_000)):
        th, ph, w = _points(N, seed)
        nb = ct.c_size_t()
        L.check(lib.dsht_workspace_size(d._plan, N, ct.byref(nb)))
        assert nb.value <= lib.dsht_noalloc_scratch_bytes()
        ref = _with_workspace(lib, d, th, ph, w)
        got = _no_alloc(lib, d, th, ph, w)
        assert np.abs(got - ref).max() <= TOL_MIXED * np.abs(ref).max()


def test_no_alloc_rejects_problems_beyond_its_scratch():
    lib = L.load()
    d = DirectSHT(600, 1200)
    th, ph, w = _points(1000, 2)
    alm = torch.empty(d.Nlm, dtype=torch.complex128, device="cuda")
    rc = lib.dsht_execute_noalloc(d._plan, L.ptr(th), L.ptr(ph), L.ptr(w), 1000, L.DSHT_MODE_CALL, L.ptr(alm),
                                  None)
    assert rc == L.DSHT_ERR_NOMEM
    assert "scratch" in L.last_error()
