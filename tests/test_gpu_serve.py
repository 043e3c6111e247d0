"""The serving loop on the GPU: Poisson arrivals of multi-map requests of mixed sizes and
(Nl, Nx), HBM-budget admission, overlapping slots.  Each request's alm in the mix must equal
the same request run alone within 1e-7 x max|alm| per map (the mixed level's tolerance)."""
import numpy as np
import pytest

from directsht_b200 import DirectSHT
from directsht_b200.batch import PlanCache
from directsht_b200.serve import GpuExecutor, Request, Server, cap_points, poisson_requests, replay
from oracle import dsht_oracle as O

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone_results():
    rng = np.random.default_rng(3)
    timed = poisson_requests(rng, 24, 2000.0, Nls=(32, 64), n_range=(2e3, 1e5), maps=(1, 4))
    cache = PlanCache(precision="mixed", compact_min_nl=64)  # Nl=64 plans keep compact tables only
    for Nl in (32, 64):
        cache.get(Nl, 2 * Nl)
    srv = Server(GpuExecutor(cache), budget_bytes=2 << 30, slots=4).start()
    futs = replay(srv, timed)
    srv.stop(drain=True, timeout=300)
    st = srv.stats()
    assert st["requests"] == len(timed) and st["rejected"] == 0
    assert st["max_concurrent"] >= 2  # requests overlapped on the device
    for (t, req), f in zip(timed, futs):
        got = f.result(timeout=1)
        alone = cache.get(*req.key).call_maps(req.theta, req.phi, req.w)
        assert got.shape == alone.shape
        for k in range(req.nmaps):
            err = np.abs(got[k] - alone[k]).max() / np.abs(alone[k]).max()
            assert err <= 1e-7, (req.rid, k, err)


def test_budget_smaller_than_mix_still_serves_everything():
    """With room for one request at a time the loop degrades to one-by-one, all served."""
    rng = np.random.default_rng(4)
    timed = poisson_requests(rng, 6, 5000.0, Nls=(32,), n_range=(5e3, 2e4), maps=(1, 2))
    cache = PlanCache(precision="mixed")
    ex = GpuExecutor(cache)
    biggest = max(ex.footprint(r) for _, r in timed)
    srv = Server(ex, budget_bytes=biggest, slots=4).start()
    futs = replay(srv, timed)
    srv.stop(drain=True, timeout=120)
    assert all(f.done() and f.exception() is None for f in futs)
    assert srv.stats()["requests"] == 6


@pytest.mark.slow
def test_served_caps_nl1024_vs_fp64_and_oracle():
    """Serving-stream requests at Nl=1024, Nx=2048 on the compact-table plan the server keeps
    resident, with points in caps of half-angle 0.2 rad (a few hundred x bins) and 0.5 rad:
    every served map within 1e-7 x max|alm| of the FP64 plan, and the transform of map 0's
    equatorial and rotated polar points against the per-m oracle."""
    rng = np.random.default_rng(7)
    Nl, Nx = 1024, 2048
    reqs = []
    for alpha, N, k in ((0.2, 300_000, 3), (0.5, 1_000_000, 2), (0.2, 50_000, 1)):
        th, ph = cap_points(rng, N, alpha)
        w = rng.uniform(0.5, 1.5, (k, N)).astype(np.float32)
        reqs.append((0.0, Request(Nl, Nx, th, ph, w)))
    cache = PlanCache(precision="mixed", compact_min_nl=1024)
    plan = cache.get(Nl, Nx)
    srv = Server(GpuExecutor(cache), budget_bytes=16 << 30, slots=4).start()
    futs = replay(srv, reqs)
    srv.stop(drain=True, timeout=600)
    fp64 = DirectSHT(Nl, Nx)
    for (_, req), f in zip(reqs, futs):
        got = f.result(timeout=1)
        for k in range(req.nmaps):
            ref = fp64(req.theta, req.phi, req.w[k].astype(np.float64))
            err = np.abs(got[k] - ref).max() / np.abs(ref).max()
            assert err <= 1e-7, (req.rid, k, err)
    del fp64
    # both point sets of the first request against the oracle (map 0)
    req = reqs[0][1]
    w0 = req.w[0].astype(np.float64)
    pol = np.abs(np.cos(req.theta)) >= 0.75
    sets = [(req.theta[~pol], req.phi[~pol], w0[~pol])]
    if pol.any():
        tr, pr = O.rotate_points(req.theta[pol], req.phi[pol])
        sets.append((tr, pr, w0[pol]))
    for t_, p_, w_ in sets:
        if len(t_) == 0:
            continue
        a = plan.basic_sht(t_, p_, w_.copy(), verbose=False)
        scale = np.abs(a).max()
        for m in (0, 3, 400, 1023):
            r0 = O.healpy_index(m, m, Nl)
            col = O.basic_sht_column(Nl, Nx, 0.75, m, t_, p_, w_)
            assert np.abs(a[r0:r0 + Nl - m] - col).max() <= 1e-7 * scale, m
