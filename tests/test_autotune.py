"""Autotuner (parallelcmacionize_b200/autotune.py): candidate set, selection,
on-disk cache; one GPU test that tunes a small grid for real."""
import json

import numpy as np
import pytest

from parallelcmacionize_b200 import GridSpec
from parallelcmacionize_b200.autotune import Autotuner, WalkConfig, cache_key, candidates
from parallelcmacionize_b200.problems import lognormal_config, lognormal_density


def test_candidates_respect_divisibility():
    c = candidates((48, 48, 48))  # 16 divides 48, 8 divides 48
    assert {x.sub_side for x in c} == {8, 16}
    c = candidates((40, 40, 40))  # only 8
    assert {x.sub_side for x in c} == {8}
    with pytest.raises(ValueError):
        candidates((12, 12, 12))
    c64 = candidates((64, 64, 64), precision="fp64")
    assert all(x.packets_per_chunk == 0 and x.max_run_chunks == 0 for x in c64)
    assert len(candidates((64, 64, 64), chunks=(64, 128), runs=(4, 16, 64))) == 2 * 2 * 3


def test_config_regrids():
    g = GridSpec(box=(0, 0, 0, 1, 1, 1), ncell=(64, 32, 128), num_subgrid=(4, 2, 8),
                 sources=[(0.5, 0.5, 0.5, 1e49)], num_photon=1000)
    h = WalkConfig(sub_side=8).grid(g)
    assert h.num_subgrid == (8, 4, 16) and h.sub_ncell == (8, 8, 8)
    assert h.sources == g.sources and h.num_photon == 1000


def _model(cfg, grid, nH, xH):
    # a smooth made-up rate with a unique best point
    return (1e10 * (2.0 if cfg.sub_side == 16 else 1.0) / (1 + abs(np.log2(cfg.packets_per_chunk / 128)))
            / (1 + 0.1 * abs(np.log2(cfg.max_run_chunks / 16))))


def test_tune_picks_best_and_caches(tmp_path):
    spec, nH = lognormal_config(ncell=32, num_subgrid=2, num_photon=100_000)
    calls = []

    def measure(cfg, grid, n, x):
        calls.append(cfg)
        assert n.shape == (32, 32, 32) and np.all(x == 1e-6)
        return _model(cfg, grid, n, x)

    path = tmp_path / "tune.json"
    t = Autotuner(cache_path=str(path), measure=measure)
    best = t.tune(spec, lognormal_density(32))
    assert best == WalkConfig(16, 128, 16, "fixed64", 0)
    n = len(calls)
    assert n == len(candidates((32, 32, 32))) and len(t.last_table) == n
    # second call: from the cache, no measurement
    assert t.tune(spec, lognormal_density(32)) == best and len(calls) == n
    d = json.loads(path.read_text())
    (key, entry), = d.items()
    assert entry["config"]["sub_side"] == 16 and entry["searched"] == n
    # another packet count -> another key
    spec2, _ = lognormal_config(ncell=32, num_subgrid=2, num_photon=10_000_000)
    assert cache_key("dev", spec, "fp32") != cache_key("dev", spec2, "fp32")
    t.tune(spec2, lognormal_density(32))
    assert len(calls) == 2 * n and len(json.loads(path.read_text())) == 2
    # force re-measures
    t.tune(spec, lognormal_density(32), force=True)
    assert len(calls) == 3 * n


def test_corrupt_cache_is_ignored(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text("{not json")
    spec, _ = lognormal_config(ncell=16, num_subgrid=1, num_photon=1000)
    t = Autotuner(cache_path=str(path), measure=_model)
    assert t.cached(spec) is None
    t.tune(spec, np.full((16, 16, 16), 1e8), configs=[WalkConfig(8, 64, 16)])
    assert t.cached(spec) == WalkConfig(8, 64, 16)


@pytest.mark.gpu
def test_autotune_on_gpu(tmp_path):
    spec, nH = lognormal_config(ncell=32, num_subgrid=2, num_photon=200_000, num_sources=2)
    cube = lognormal_density(32, seed=42)
    t = Autotuner(cache_path=str(tmp_path / "t.json"), iterations=2, warmup=1)
    cfgs = [WalkConfig(8, 64, 16), WalkConfig(16, 128, 64)]
    best = t.tune(spec, cube, configs=cfgs)
    assert best in cfgs and all(r > 0 for _, r in t.last_table)
    eng, cfg = t.engine(spec, cube)
    assert cfg == best and eng.grids[0].sub_ncell == (best.sub_side,) * 3
    st = eng.run_iterations(2, seed=3)
    assert all(s[0]["error_flags"] == 0 for s in st)
    eng.close()


def test_tune_batch_by_class_then_chunking(tmp_path):
    """The batch search: the untuned start first, then the subgrid side of
    each size class (largest class first), then the context's chunking; every
    step keeps the best so far; the result is cached by the batch's classes."""
    from parallelcmacionize_b200.autotune import BatchConfig, batch_cache_key
    from parallelcmacionize_b200.problems import batch_configs
    cfgs = batch_configs(count=6, select=set())
    grids = [g for g, _ in cfgs]
    fields = [None] * len(grids)
    classes = sorted({"x".join(map(str, g.ncell)) for g in grids},
                     key=lambda n: -int(n.split("x")[0]))

    def model(cfg, gs, fs):
        # 8^3 subgrids win for grids of 64 cells or fewer per axis, 16^3 above;
        # 64-packet chunks and 16-chunk claims win
        r = 1e10
        for name, side in cfg.sides:
            small = int(name.split("x")[0]) <= 64
            r *= 1.1 if (side == 8) == small else 1.0
        r /= 1 + abs(np.log2(cfg.packets_per_chunk / 64))
        r /= 1 + 0.1 * abs(np.log2(cfg.max_run_chunks / 16))
        return r

    calls = []

    def measure(cfg, gs, fs):
        calls.append(cfg)
        assert gs is grids and fs is fields
        return model(cfg, gs, fs)

    t = Autotuner(cache_path=str(tmp_path / "t.json"), measure=None)
    best = t.tune_batch(grids, fields, measure=measure)
    assert calls[0] == BatchConfig(sides=tuple((c, 16) for c in classes))
    assert dict(best.sides) == {c: (8 if int(c.split("x")[0]) <= 64 else 16) for c in classes}
    assert (best.packets_per_chunk, best.max_run_chunks) == (64, 16)
    assert len(t.last_table) == len(calls) == 1 + len(classes) + 3 * 2 - 1
    n = len(calls)
    assert t.tune_batch(grids, fields, measure=measure) == best and len(calls) == n
    key = batch_cache_key("cuda0", grids, "fp32")
    assert "|batch|" in key and all(c in key for c in classes)
    # regridding keeps every instance's box, sources and budget
    for g0, g in zip(grids, best.grids(grids)):
        assert g.ncell == g0.ncell and g.sources == g0.sources
        assert g.num_photon == g0.num_photon
        assert g.sub_ncell[0] == best.side_of(g0)
