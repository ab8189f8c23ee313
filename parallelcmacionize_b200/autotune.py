"""Autotuner for the transport's launch shape (no reference counterpart).

The reference fixes its subgrid decomposition and buffer sizes in the
parameter file (params.txt: ``num_subgrid``, ``PHOTONBUFFER_SIZE`` in
PhotonBuffer.hpp:34).  On the GPU those choices set how many cells a CTA
stages in shared memory, how many CTAs fit on an SM and how often a CTA flushes
its tallies, and the best choice depends on the grid, the source layout and the
packet count.  ``Autotuner`` times a short run of each candidate and keeps the
fastest, cached on disk by device, grid shape, precision and packet count.

A candidate (``WalkConfig``) chooses:

* ``sub_side``          -- cells per subgrid along each axis (8 or 16 by
  default); the grid is re-blocked for it,
* ``packets_per_chunk`` -- packets a CTA takes per claim (the packet ring slot),
* ``max_run_chunks``    -- most chunks claimed at once: how long a CTA stays on
  one subgrid before it flushes its shared tallies to J,
* ``refill_lanes``      -- lanes a warp lets go idle before it routes finished
  packets and refills them in one batch,
* ``tally``             -- shared-memory tally form of the FP32 walk,
* ``ctas_per_sm``       -- 0 = the engine's occupancy choice.

The subgrid decomposition changes where the FP32 walk re-anchors its
positions, so results of two candidates agree to FP32 rounding, not bit for
bit; every candidate is a correct transport.

A batch of independent instances of uneven size (one context, one launch per
kernel; ``Autotuner.tune_batch``) is tuned as a whole, since an instance's
rate alone says little about the batch: the subgrid side of each size class
first (greedy, class by class, largest first), then the chunking shared by
the context (``BatchConfig``).
"""
from __future__ import annotations

import json
import math
import os
import tempfile
import time
from collections import Counter
from dataclasses import asdict, dataclass, replace

import numpy as np

from .engine import GridSpec, TransportEngine, blocked_to_cube, cube_to_blocked


@dataclass(frozen=True)
class WalkConfig:
    sub_side: int = 16
    packets_per_chunk: int = 128
    max_run_chunks: int = 64
    tally: str = "fixed64"
    ctas_per_sm: int = 0
    refill_lanes: int = 16

    def grid(self, base: GridSpec) -> GridSpec:
        """``base`` re-decomposed into subgrids of ``sub_side`` cells per axis."""
        nsub = tuple(int(n) // self.sub_side for n in base.ncell)
        return GridSpec(box=base.box, ncell=base.ncell, num_subgrid=nsub,
                        recombination_rate=base.recombination_rate,
                        cross_section=base.cross_section, sources=list(base.sources),
                        num_photon=base.num_photon,
                        reemission_probability=base.reemission_probability)

    def engine_options(self) -> dict:
        return dict(packets_per_chunk=self.packets_per_chunk, tally=self.tally,
                    ctas_per_sm=self.ctas_per_sm, max_run_chunks=self.max_run_chunks,
                    refill_lanes=self.refill_lanes)


@dataclass(frozen=True)
class BatchConfig:
    """Launch shape of a batch: ``sides`` maps each size class (cells per axis,
    "NxNxN") to its subgrid side; the rest is shared by the context."""
    sides: tuple = ()  # (("32x32x32", 16), ...)
    packets_per_chunk: int = 128
    max_run_chunks: int = 64
    tally: str = "fixed64"
    ctas_per_sm: int = 0
    refill_lanes: int = 16

    def side_of(self, grid: GridSpec) -> int:
        return dict(self.sides).get(_class_name(grid), 16)

    def grids(self, base_grids):
        return [WalkConfig(sub_side=self.side_of(g)).grid(g) for g in base_grids]

    def engine_options(self) -> dict:
        return dict(packets_per_chunk=self.packets_per_chunk, tally=self.tally,
                    ctas_per_sm=self.ctas_per_sm, max_run_chunks=self.max_run_chunks,
                    refill_lanes=self.refill_lanes)


def _class_name(grid: GridSpec) -> str:
    return "x".join(str(int(v)) for v in grid.ncell)


def reblock(nH_blocked, old: GridSpec, new: GridSpec):
    """A blocked field of ``old`` in the subgrid decomposition of ``new``."""
    cube = blocked_to_cube(nH_blocked, old.ncell, old.num_subgrid)
    return cube_to_blocked(cube, new.ncell, new.num_subgrid)


def candidates(ncell, precision="fp32", sides=(8, 16), chunks=(64, 128, 256),
               runs=(16, 64), tallies=("fixed64",), ctas=(0,), refills=(16,)):
    """Every valid combination for a grid of ``ncell`` cells per axis.

    A side must divide every axis.  The FP64 walk has no shared tallies and no
    packet ring, so only the decomposition is searched for it.
    """
    ncell = tuple(int(n) for n in ncell)
    ok_sides = [s for s in sides if all(n % s == 0 for n in ncell)]
    if not ok_sides:
        raise ValueError(f"no subgrid side of {sides} divides the grid {ncell}")
    if precision == "fp64":
        return [WalkConfig(sub_side=s, packets_per_chunk=0, max_run_chunks=0, tally="fixed64",
                           ctas_per_sm=0) for s in ok_sides]
    return [WalkConfig(s, c, r, t, k, f) for s in ok_sides for c in chunks for r in runs
            for t in tallies for k in ctas for f in refills]


def default_cache_path() -> str:
    p = os.environ.get("CMI_AUTOTUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "parallelcmacionize_b200",
                        "autotune.json")


def cache_key(device_name: str, grid: GridSpec, precision: str) -> str:
    """Grid shape, source count and packet count to the nearest power of two."""
    bucket = int(round(math.log2(max(1, int(grid.num_photon)))))
    n = "x".join(str(int(v)) for v in grid.ncell)
    return f"{device_name}|{n}|src{len(grid.sources)}|pk2^{bucket}|{precision}"


def batch_cache_key(device_name: str, grids, precision: str) -> str:
    """Size classes with their counts, total packets to the nearest power of two."""
    classes = sorted(Counter(_class_name(g) for g in grids).items())
    total = sum(int(g.num_photon) for g in grids)
    bucket = int(round(math.log2(max(1, total))))
    cls = ",".join(f"{n}*{k}" for n, k in classes)
    return f"{device_name}|batch|{cls}|pk2^{bucket}|{precision}"


def _device_name(device: int) -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(device).replace("|", "/")
    except Exception:
        pass
    return f"cuda{device}"


class Autotuner:
    """Pick the fastest ``WalkConfig`` for a grid by timing short runs.

    ``measure(config, grid, nH_cube, xH_cube) -> crossings per second`` may be
    replaced (tests use a model of it); the default builds an engine for the
    candidate, runs ``warmup`` untimed and ``iterations`` timed iterations of
    the transport + balance loop from the same initial fields and divides the
    cell crossings by the time between two device synchronisations.
    """

    def __init__(self, cache_path=None, device=0, precision="fp32", iterations=2, warmup=1,
                 seed=42, measure=None):
        self.cache_path = cache_path or default_cache_path()
        self.device = device
        self.precision = precision
        self.iterations = int(iterations)
        self.warmup = int(warmup)
        self.seed = int(seed)
        self.measure = measure or self._measure
        self.last_table = []

    # ---- cache ----
    def _load(self) -> dict:
        try:
            with open(self.cache_path) as f:
                d = json.load(f)
            return d if isinstance(d, dict) else {}
        except (OSError, ValueError):
            return {}

    def _store(self, key: str, entry: dict):
        d = self._load()
        d[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(self.cache_path)), exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=os.path.dirname(os.path.abspath(self.cache_path)),
                                   suffix=".tmp")
        with os.fdopen(fd, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def cached(self, grid: GridSpec):
        e = self._load().get(cache_key(_device_name(self.device), grid, self.precision))
        return WalkConfig(**e["config"]) if e else None

    # ---- search ----
    def _measure(self, cfg: WalkConfig, grid: GridSpec, nH_cube, xH_cube) -> float:
        g = cfg.grid(grid)
        with TransportEngine(g, precision=self.precision, device=self.device,
                             **cfg.engine_options()) as eng:
            nH = cube_to_blocked(nH_cube, g.ncell, g.num_subgrid)
            xH = cube_to_blocked(xH_cube, g.ncell, g.num_subgrid)
            eng.set_fields(0, nH, xH)
            if self.warmup:
                eng.run_iterations(self.warmup, seed=self.seed)
            eng.set_fields(0, nH, xH)
            eng.synchronize()
            t0 = time.perf_counter()
            st = eng.run_iterations(self.iterations, seed=self.seed + 1)
            eng.synchronize()
            dt = time.perf_counter() - t0
        crossings = sum(s[0]["cell_crossings"] for s in st)
        return crossings / dt

    def tune(self, grid: GridSpec, nH_cube, xH_cube=None, configs=None, force=False):
        """Best config for ``grid`` (from the cache unless ``force``).

        ``nH_cube``/``xH_cube`` are (nx, ny, nz) cubes; xH defaults to the
        reference's initial 1e-6 (DensitySubGrid.hpp:544-551).
        """
        key = cache_key(_device_name(self.device), grid, self.precision)
        if not force:
            hit = self._load().get(key)
            if hit:
                self.last_table = []
                return WalkConfig(**hit["config"])
        nH_cube = np.asarray(nH_cube, dtype=np.float64).reshape(tuple(grid.ncell))
        xH_cube = (np.full_like(nH_cube, 1.0e-6) if xH_cube is None
                   else np.asarray(xH_cube, dtype=np.float64).reshape(nH_cube.shape))
        configs = list(configs) if configs is not None else candidates(grid.ncell,
                                                                         self.precision)
        if not configs:
            raise ValueError("no candidate configurations")
        table = []
        for cfg in configs:
            table.append((cfg, float(self.measure(cfg, grid, nH_cube, xH_cube))))
        best, rate = max(table, key=lambda t: t[1])
        self.last_table = table
        self._store(key, {"config": asdict(best), "crossings_per_s": rate,
                          "searched": len(table)})
        return best

    # ---- batches ----
    def _measure_batch(self, cfg: BatchConfig, grids, fields) -> float:
        gs = cfg.grids(grids)
        with TransportEngine(gs, precision=self.precision, device=self.device,
                             **cfg.engine_options()) as eng:
            for i, (g0, g, n) in enumerate(zip(grids, gs, fields)):
                eng.set_fields(i, reblock(n, g0, g), np.full(n.size, 1.0e-6))
            if self.warmup:
                eng.run_iterations(self.warmup, seed=self.seed)
            for i, n in enumerate(fields):
                eng.set_fields(i, None, np.full(n.size, 1.0e-6))
            eng.synchronize()
            t0 = time.perf_counter()
            st = eng.run_iterations(self.iterations, seed=self.seed + 1)
            eng.synchronize()
            dt = time.perf_counter() - t0
        return sum(s["cell_crossings"] for it in st for s in it) / dt

    def tune_batch(self, grids, fields, sides=(8, 16), chunks=(64, 128, 256), runs=(16, 64),
                   force=False, measure=None):
        """Best ``BatchConfig`` for a batch of ``grids`` with blocked n_H ``fields``
        (in the grids' own decomposition), from the cache unless ``force``.
        ``self.last_table`` lists every measured (config, crossings/s); its first
        entry is the untuned start: every class in 16^3 subgrids, 128-packet
        chunks, 64-chunk claims."""
        measure = measure or self._measure_batch
        key = batch_cache_key(_device_name(self.device), grids, self.precision)
        if not force:
            hit = self._load().get(key)
            if hit:
                self.last_table = []
                c = hit["config"]
                return BatchConfig(**dict(c, sides=tuple(tuple(x) for x in c["sides"])))
        classes = sorted({_class_name(g) for g in grids},
                         key=lambda n: -int(n.split("x")[0]))
        ok = {c: [s for s in sides if all(int(v) % s == 0 for v in c.split("x"))]
              for c in classes}
        table = []
        rates = {}

        def rate_of(cand):
            if cand not in rates:
                rates[cand] = float(measure(cand, grids, fields))
                table.append((cand, rates[cand]))
            return rates[cand]

        best = BatchConfig(sides=tuple((c, 16 if 16 in ok[c] else ok[c][0]) for c in classes))
        rate = rate_of(best)
        for c in classes:  # the subgrid side, one size class at a time
            for s in ok[c]:
                cand = replace(best, sides=tuple((k, s if k == c else v) for k, v in best.sides))
                r = rate_of(cand)
                if r > rate:
                    best, rate = cand, r
        for ch in chunks:  # then the chunking shared by the context
            for ru in runs:
                cand = replace(best, packets_per_chunk=ch, max_run_chunks=ru)
                r = rate_of(cand)
                if r > rate:
                    best, rate = cand, r
        self.last_table = table
        self._store(key, {"config": asdict(best), "crossings_per_s": rate,
                          "untuned_crossings_per_s": table[0][1], "searched": len(table)})
        return best

    def engine(self, grid: GridSpec, nH_cube, xH_cube=None, **engine_kw):
        """A ``TransportEngine`` for ``grid`` in the tuned decomposition, with
        the fields set; returns (engine, config).  Fields read back from it are
        in that decomposition's blocked order (``blocked_to_cube`` with
        ``engine.grids[0]``)."""
        cfg = self.tune(grid, nH_cube, xH_cube)
        g = cfg.grid(grid)
        kw = cfg.engine_options()
        kw.update(engine_kw)
        eng = TransportEngine(g, precision=self.precision, device=self.device, **kw)
        nH = cube_to_blocked(np.asarray(nH_cube, np.float64).reshape(tuple(g.ncell)), g.ncell,
                             g.num_subgrid)
        xH = (np.full(nH.size, 1.0e-6) if xH_cube is None else
              cube_to_blocked(np.asarray(xH_cube, np.float64).reshape(tuple(g.ncell)),
                              g.ncell, g.num_subgrid))
        eng.set_fields(0, nH, xH)
        return eng, cfg
