"""The serving loop on the GPU: Poisson arrivals of multi-map requests of mixed sizes and
(Nl, Nx), HBM-budget admission, overlapping slots.  Each request's alm in the mix must equal
the same request run alone within 1e-7 x max|alm| per map (the mixed level's tolerance)."""
import numpy as np
import pytest

from directsht_b200.batch import PlanCache
from directsht_b200.serve import GpuExecutor, Server, poisson_requests, replay

pytestmark = pytest.mark.gpu


def test_served_results_equal_alone_results():
    rng = np.random.default_rng(3)
    timed = poisson_requests(rng, 24, 2000.0, Nls=(32, 64), n_range=(2e3, 1e5), maps=(1, 4))
    cache = PlanCache(precision="mixed", f32_tables_min_nl=64)  # Nl=64 plans keep FP32 tables only
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
