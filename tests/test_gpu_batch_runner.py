"""The uneven-batch runner (directsht_b200.batch): mixed (Nl, Nx) and sizes, sub-batch
streams, CUDA-graph capture and the autotuner.  Every transform must equal its own single
call (bit for bit on the mixed path when every bin fits one piece, 1e-13 otherwise)."""
import numpy as np
import pytest
import torch

from directsht_b200.batch import PlanCache, TransformBatch, autotune

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _transforms(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        Nl = int(rng.choice([16, 32, 64]))
        N = int(np.exp(rng.uniform(np.log(10), np.log(30000))))
        th = np.arccos(rng.uniform(-1, 1, N))
        ph = rng.uniform(0, 2 * np.pi, N)
        w = rng.uniform(0.5, 1.5, N)
        out.append((Nl, 2 * Nl, th, ph, w))
    return out


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_runner_matches_single_calls(precision):
    ts = _transforms(1, 14)
    cache = PlanCache(precision=precision)
    cfg = {}
    for k in {(t[0], t[1], 0.75) for t in ts}:
        cfg[k] = {"streams": 2, "piece_max": 512, "maps_per_pass": 2 if precision == "mixed" else 0}
    b = TransformBatch(cache, ts, config=cfg)
    b.run()
    torch.cuda.synchronize()
    b.check()
    for i, t in enumerate(ts):
        single = cache.get(t[0], t[1])(t[2], t[3], t[4])
        assert _rel(b.alms[i].cpu().numpy(), single) <= 1e-13, i
    # the captured graph gives the same numbers on every replay
    ref = [a.clone() for a in b.alms]
    b.capture()
    for _ in range(2):
        for a in b.alms:
            a.zero_()
        b.run()
        torch.cuda.synchronize()
        b.check()
        for i in range(len(ts)):
            assert torch.equal(b.alms[i], ref[i]) or _rel(b.alms[i].cpu().numpy(), ref[i].cpu().numpy()) <= 1e-13
    b.release()


def test_autotune_picks_and_caches(tmp_path):
    ts = _transforms(2, 6)
    cache = PlanCache(precision="mixed")
    b = TransformBatch(cache, ts)
    path = str(tmp_path / "tune.json")
    cfg = autotune(b, path=path, reps=1)
    assert set(cfg) == set(b.groups)
    for c in cfg.values():
        assert c["piece_max"] in (0, 512, 1024, 2048, 4096, 16384) and c["streams"] >= 1
    cfg2 = autotune(b, path=path)  # served from the cache
    assert cfg2 == cfg
    b.run()
    torch.cuda.synchronize()
    b.check()
    for i, t in enumerate(ts):
        assert _rel(b.alms[i].cpu().numpy(), cache.get(t[0], t[1])(t[2], t[3], t[4])) <= 1e-13
