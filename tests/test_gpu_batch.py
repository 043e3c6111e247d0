"""Batches of independent transforms on one plan (dsht_execute_batch / dsht_enqueue_batch).

Each transform of a batch must give the alm of its own single call: bit for bit on the
mixed path when every bin fits one piece (integer bin sums are exact, and the order of the
remaining arithmetic is the same), within 1e-13 x max|alm| on the FP64 path (the order of
the points inside a bin varies from run to run)."""
import ctypes as ct

import numpy as np
import pytest
import torch

from directsht_b200 import DirectSHT
from directsht_b200 import _lib as L
from oracle import dsht_oracle as O

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def _sets(seed, sizes, equatorial=()):
    rng = np.random.default_rng(seed)
    out = []
    for i, n in enumerate(sizes):
        lim = 0.7 if i in equatorial else 1.0
        th = np.arccos(rng.uniform(-lim, lim, n))
        ph = rng.uniform(0, 2 * np.pi, n)
        w = rng.uniform(0.5, 1.5, n)
        out.append((th, ph, w))
    return out


SIZES = [5000, 0, 300, 40000, 1, 2500, 70000, 1200, 9000, 3]


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_f64_tables"])
def test_batch_equals_single_calls(precision):
    Nl, Nx = 64, 128
    sets = _sets(1, SIZES, equatorial=(3, 8))
    d = DirectSHT(Nl, Nx, precision=precision)
    got = d.call_batch(sets)
    tab = O.build_tables(Nl, Nx)
    for i, (th, ph, w) in enumerate(sets):
        single = d(th, ph, w)
        # the NUFFT and tensor-core bin sums (from 28 points per bin key on average) are exact
        # integer sums, so a batch item repeats its single call bit for bit; the FP64 sums
        # (fp64 level, transforms under 1024 points, sparse transforms) add in the sort's order
        if precision == "fp64" or len(th) < 28 * 4 * (Nx - 1):
            assert _rel(got[i], single) <= 1e-13 or not np.any(single), i
        else:
            assert np.array_equal(got[i], single), i
        if len(th):
            assert _rel(got[i], O.direct_sht(tab, th, ph, w)) <= (1e-12 if precision == "fp64" else 1e-7), i


def test_batch_basic_mode_and_errors():
    d = DirectSHT(32, 64)
    sets = _sets(2, [400, 900], equatorial=(0, 1))
    got = d.call_batch(sets, mode="basic")
    tab = O.build_tables(32, 64)
    for i, (th, ph, w) in enumerate(sets):
        assert _rel(got[i], O.basic_sht(tab, th, ph, w)) <= 1e-12
    bad = _sets(3, [100, 100], equatorial=(0,))  # set 1 has polar points
    with pytest.raises(AssertionError):
        d.call_batch(bad, mode="basic")
    with pytest.raises(ValueError):
        d.call_batch([(np.zeros(0), np.zeros(0), np.zeros(0))], mode="basic")


def test_enqueue_batch_status_words():
    """Per-transform flags: a basic-mode batch with one out-of-range set reports it alone."""
    d = DirectSHT(32, 64)
    sets = _sets(4, [500, 500, 500], equatorial=(0, 2))
    dev = [tuple(torch.tensor(a, device="cuda") for a in s) for s in sets]
    alms = [torch.empty(d.Nlm, dtype=torch.complex128, device="cuda") for _ in sets]
    n = len(sets)
    arr = lambda xs: (ct.c_void_p * n)(*[x.data_ptr() for x in xs])
    Ns = (ct.c_int64 * n)(*[len(s[0]) for s in sets])
    status = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    nb = ct.c_size_t()
    L.check(d._lib.dsht_workspace_size_batch(d._plan, 500, n, ct.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    L.check(d._lib.dsht_enqueue_batch(d._plan, n, arr([x[0] for x in dev]), arr([x[1] for x in dev]),
                                      arr([x[2] for x in dev]), Ns, L.DSHT_MODE_BASIC, arr(alms), L.ptr(status),
                                      L.ptr(ws), ws.numel(), ct.c_void_p(s)))
    codes = [d._lib.dsht_status(int(f) & 0xffffffff, L.DSHT_MODE_BASIC) for f in status.cpu().numpy()]
    assert codes == [L.DSHT_OK, L.DSHT_ERR_THETA_RANGE, L.DSHT_OK]
    # the enqueued call needs a caller workspace
    assert d._lib.dsht_enqueue_batch(d._plan, n, arr([x[0] for x in dev]), arr([x[1] for x in dev]),
                                     arr([x[2] for x in dev]), Ns, L.DSHT_MODE_BASIC, arr(alms), None, None, 0,
                                     ct.c_void_p(s)) == L.DSHT_ERR_INVALID


def test_stage_times_of_an_enqueued_batch():
    """dsht_profile_read adds the stage events of the last dsht_enqueue_batch call once its
    stream has finished: every stage of a mixed batch with polar points is timed, once."""
    d = DirectSHT(64, 128, precision="mixed")
    sets = _sets(6, [40000, 30000, 50000])
    dev = [tuple(torch.tensor(a, device="cuda") for a in s) for s in sets]
    alms = [torch.empty(d.Nlm, dtype=torch.complex128, device="cuda") for _ in sets]
    n = len(sets)
    arr = lambda xs: (ct.c_void_p * n)(*[x.data_ptr() for x in xs])
    Ns = (ct.c_int64 * n)(*[len(s[0]) for s in sets])
    nb = ct.c_size_t()
    L.check(d._lib.dsht_workspace_size_batch(d._plan, 50000, n, ct.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    s = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    ms = (ct.c_double * 5)()
    calls = ct.c_int64()
    L.check(d._lib.dsht_profile_enable(d._plan, 1))
    L.check(d._lib.dsht_profile_read(d._plan, ms, ct.byref(calls), 1))
    L.check(d._lib.dsht_enqueue_batch(d._plan, n, arr([x[0] for x in dev]), arr([x[1] for x in dev]),
                                      arr([x[2] for x in dev]), Ns, L.DSHT_MODE_CALL, arr(alms), None,
                                      L.ptr(ws), ws.numel(), s))
    torch.cuda.synchronize()
    L.check(d._lib.dsht_profile_read(d._plan, ms, ct.byref(calls), 1))
    L.check(d._lib.dsht_profile_enable(d._plan, 0))
    assert calls.value == 1
    assert all(v > 0.0 for v in ms), list(ms)
    # read again: nothing new was enqueued, nothing is added twice
    L.check(d._lib.dsht_profile_read(d._plan, ms, ct.byref(calls), 0))
    assert calls.value == 0 and all(v == 0.0 for v in ms)
    for (th, ph, w), a in zip(sets, alms):
        ref = O.direct_sht(O.build_tables(64, 128), th, ph, w)
        assert _rel(a.cpu().numpy(), ref) <= 1e-7


def test_enqueue_batch_in_cuda_graph():
    """The enqueued batch captures into a CUDA graph; replays give the eager results."""
    Nl, Nx = 48, 96
    d = DirectSHT(Nl, Nx, precision="mixed")
    sets = _sets(5, [3000, 20000, 500, 8000])
    eager = d.call_batch(sets)
    dev = [tuple(torch.tensor(a, device="cuda") for a in s) for s in sets]
    n = len(sets)
    alms = [torch.zeros(d.Nlm, dtype=torch.complex128, device="cuda") for _ in sets]
    arr = lambda xs: (ct.c_void_p * n)(*[x.data_ptr() for x in xs])
    Ns = (ct.c_int64 * n)(*[len(s[0]) for s in sets])
    status = torch.zeros(n, dtype=torch.int32, device="cuda")
    nb = ct.c_size_t()
    L.check(d._lib.dsht_workspace_size_batch(d._plan, max(Ns), n, ct.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # warm-up outside capture (sets kernel attributes)
        L.check(d._lib.dsht_enqueue_batch(d._plan, n, arr([x[0] for x in dev]), arr([x[1] for x in dev]),
                                          arr([x[2] for x in dev]), Ns, L.DSHT_MODE_CALL, arr(alms), L.ptr(status),
                                          L.ptr(ws), ws.numel(), ct.c_void_p(side.cuda_stream)))
    torch.cuda.current_stream().wait_stream(side)
    with torch.cuda.graph(g):
        L.check(d._lib.dsht_enqueue_batch(d._plan, n, arr([x[0] for x in dev]), arr([x[1] for x in dev]),
                                          arr([x[2] for x in dev]), Ns, L.DSHT_MODE_CALL, arr(alms), L.ptr(status),
                                          L.ptr(ws), ws.numel(),
                                          ct.c_void_p(torch.cuda.current_stream().cuda_stream)))
    for _ in range(2):
        for a in alms:
            a.zero_()
        g.replay()
        torch.cuda.synchronize()
        for i in range(n):  # under 28 points per bin key the FP64 bin sums run: their order varies
            got = alms[i].cpu().numpy()
            exact = len(sets[i][0]) >= 28 * 4 * (Nx - 1)
            assert np.array_equal(got, eager[i]) if exact else _rel(got, eager[i]) <= 1e-13
    assert all(d._lib.dsht_status(int(f), L.DSHT_MODE_CALL) == L.DSHT_OK for f in status.cpu().numpy())


def test_compact_table_plan():
    """A plan holding the compact (4-byte fixed-point digit) tables only: mixed results
    within 1e-7 of the oracle, small transforms included (FP64 bin sums on the digit
    tables); its rows are the FP64 rows to within 2^-31 of the row's scale."""
    Nl, Nx = 64, 128
    d = DirectSHT(Nl, Nx, compact_tables=True)
    assert d.precision == "mixed"
    with pytest.raises(Exception):
        d.set_precision("fp64")
    tab = O.build_tables(Nl, Nx)
    d64 = DirectSHT(Nl, Nx)
    dx = 0.75 / (Nx - 1)
    for l, m in ((10, 3), (63, 0), (40, 40), (0, 0), (1, 0)):
        yv, yd = d64.get_Ylm(l, m), d64.get_dYlm(l, m)
        scale = max(np.abs(yv).max(), dx * np.abs(yd).max())
        assert np.abs(d.get_Ylm(l, m) - yv).max() <= 2.0 ** -30 * scale, (l, m)
        assert np.abs(d.get_dYlm(l, m) - yd).max() <= 2.0 ** -30 * scale / dx, (l, m)
    sets = _sets(6, [50000, 700, 20000])
    got = d.call_batch(sets)
    for i, (th, ph, w) in enumerate(sets):
        ref = O.direct_sht(tab, th, ph, w)
        assert _rel(got[i], ref) <= 1e-7, i
        assert _rel(d(th, ph, w), ref) <= 1e-7, i


def test_pipeline_overlapped_host_transforms():
    """Pipeline: host point sets in, host alm out, copies overlapped with the previous
    transform's kernels; every result equals DirectSHT.__call__ on the same arrays."""
    from directsht_b200.pipeline import Pipeline
    Nl, Nx = 64, 128
    d = DirectSHT(Nl, Nx, precision="mixed")
    sets = _sets(7, [30000, 12000, 30000, 500, 25000])
    pipe = Pipeline(d, max_N=30000, depth=2)
    tickets = [pipe.submit(*s) for s in sets[:2]]
    outs = [pipe.result(tickets[0])]
    tickets = tickets[1:] + [pipe.submit(*s) for s in sets[2:]]
    outs += [pipe.result(t) for t in tickets]
    for (th, ph, w), got in zip(sets, outs):
        single = d(th, ph, w)
        assert _rel(got, single) <= 1e-13 or np.array_equal(got, single)
    with pytest.raises(ValueError):
        pipe.submit(*_sets(8, [40000])[0])
    # pinned CPU tensors go to the device without the staging copy
    th, ph, w = sets[0]
    pt = [torch.from_numpy(a).pin_memory() for a in (th, ph, w)]
    assert _rel(pipe.result(pipe.submit(*pt)), outs[0]) <= 1e-13
