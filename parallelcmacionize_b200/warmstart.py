"""Learned warm start for the plain method (no reference counterpart).

The reference starts every photoionization run from x_H = 1e-6 everywhere
(DensitySubGrid.hpp:544-551) and iterates.  Here a small 3D convolutional
U-Net (the CUDA library's cmi_unet_*: BF16 tensor-core convolutions with FP32
accumulation, trained by the library's own backward kernels) predicts log10
x_H from [log10 n_H, log10 of the source flux sum_i L_i / (4 pi r_i^2)], and
the plain iteration starts from that field.  The Monte Carlo iteration still
decides convergence (cmi_run_until_converged); the network only chooses where
it starts, so a bad prediction costs iterations, never correctness.

* ``UNet``             -- the network (create, parameters, forward,
  gradients, Adam step, features, save / load).
* ``generate_runs``    -- training data: batched plain-method runs of the
  log-normal generator, iterated to convergence; the label is log10 of x_H
  averaged over the last iterations (less Monte Carlo noise).
* ``train``            -- Adam on mean squared error of log10 x_H.
* ``generate_large_runs`` / ``train_crops`` -- the same for the 256^3
  generator (problems.large_config): long plain runs kept on the device,
  training on random 64^3 windows, fine-tuned from the 64^3 weights with an
  asymmetric loss (``UNet.set_loss_weight``) that penalises predicting x_H too
  high: an ionization front predicted too far in towards the source moves out
  by about one cell per plain iteration (one neutral cell is tens of optical
  depths), while one predicted too far out is pulled back in one iteration.
* ``weights_for``      -- the shipped weights for a grid: trained at its own
  side if there are such (256^3), else the 64^3 network, which predicts finer
  grids on block-averaged n_H.
* ``warm_start``       -- features -> prediction -> x_H of an engine instance.
* ``time_to_converge`` -- iterations and wall time to convergence from the
  plain start and from the warm start, on the same inputs.

Device memory is handled with torch tensors (CUDA); the arithmetic is the
library's.  Run ``python -m parallelcmacionize_b200.warmstart --help`` for the
training pipeline that produced the shipped weights.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import _lib
from ._lib import check_unet

# log10 x_H below this is not predicted (the plain start is 1e-6)
LOG10_XH_MIN = -8.0
NUM_FEATURES = 3  # density, unattenuated flux, Stromgren ratio (cmi_unet_features)
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "warmstart_unet64.npz")
LARGE_WEIGHTS = os.path.join(WEIGHTS_DIR, "warmstart_unet256.npz")
# grid side -> shipped weights trained at that side
SHIPPED = {64: DEFAULT_WEIGHTS, 256: LARGE_WEIGHTS}


def weights_for(grid):
    """Shipped weights for ``grid``: the network trained on grids of its side
    when there is one, else the 64^3 network."""
    n = tuple(int(v) for v in grid.ncell)
    if n[0] == n[1] == n[2] and n[0] in SHIPPED and os.path.exists(SHIPPED[n[0]]):
        return SHIPPED[n[0]]
    return DEFAULT_WEIGHTS


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _dims(ncell):
    n = tuple(int(v) for v in ncell)
    return (C.c_int32 * 3)(n[2], n[1], n[0])  # network X = iz (fastest), Z = ix


class UNet:
    """The warm-start network on one GPU."""

    def __init__(self, channels=(12, 24, 48), slope=0.1, device=0, seed=0):
        self._L = _lib.load()
        cfg = _lib.UNetConfig()
        self._L.cmi_unet_default_config(C.byref(cfg))
        for k in range(3):
            cfg.channels[k] = int(channels[k])
        cfg.leaky_slope = float(slope)
        cfg.device = int(device)
        h = C.c_void_p()
        check_unet(self._L.cmi_unet_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.channels = tuple(int(c) for c in channels)
        self.slope = float(slope)
        self.device = int(device)
        n = C.c_int64()
        check_unet(self._L.cmi_unet_num_params(self._h, C.byref(n)))
        self.num_params = int(n.value)
        # feature normalisation: (mean, scale) of each of the three channels
        self.norm = np.array([8.0, 1.0, 13.0, 1.5, 0.0, 3.0], dtype=np.float32)
        self.set_params(self.initial_params(seed))

    # ---- lifetime ----
    def close(self):
        if getattr(self, "_h", None):
            self._L.cmi_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- parameters ----
    def layer_shapes(self):
        c1, c2, c3 = self.channels
        convs = [(c1, NUM_FEATURES), (c1, c1), (c2, c1), (c2, c2), (c3, c2), (c3, c3),
                 (c2, c3 + c2),
                 (c2, c2), (c1, c2 + c1), (c1, c1)]
        return convs

    def initial_params(self, seed=0):
        """He-normal convolution weights, zero biases."""
        rng = np.random.default_rng(seed)
        parts = []
        for cout, cin in self.layer_shapes():
            parts.append(rng.normal(0.0, np.sqrt(2.0 / (27 * cin)), cout * 27 * cin))
            parts.append(np.zeros(cout))
        c1 = self.channels[0]
        parts.append(rng.normal(0.0, np.sqrt(1.0 / c1), c1))
        parts.append(np.zeros(1))
        p = np.concatenate(parts).astype(np.float32)
        assert p.size == self.num_params
        return p

    def get_params(self):
        p = np.empty(self.num_params, dtype=np.float32)
        check_unet(self._L.cmi_unet_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params:
            raise ValueError(f"expected {self.num_params} parameters, got {p.size}")
        check_unet(self._L.cmi_unet_set_params(self._h, p.ctypes.data))

    def save(self, path, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez_compressed(path, params=self.get_params(), channels=np.array(self.channels),
                            slope=np.array(self.slope), norm=self.norm,
                            **{k: np.asarray(v) for k, v in meta.items()})

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS, device=0):
        d = np.load(path)
        net = cls(channels=tuple(int(c) for c in d["channels"]), slope=float(d["slope"]),
                  device=device)
        net.set_params(d["params"])
        net.norm = d["norm"].astype(np.float32)
        net.meta = {k: d[k] for k in d.files if k not in ("params", "channels", "slope", "norm")}
        return net

    # ---- compute (torch CUDA tensors, float32, cube order) ----
    # The library runs on its own stream and returns when that stream is done;
    # inputs written by torch (its own stream) are made complete first.
    def _sync(self):
        import torch
        torch.cuda.synchronize(self.device)

    def forward(self, features, ncell):
        """features [B, cells, 3] -> predicted log10 x_H [B, cells]."""
        import torch
        self._sync()
        B = features.shape[0]
        pred = torch.empty(features.shape[:2], dtype=torch.float32, device=features.device)
        check_unet(self._L.cmi_unet_forward(self._h, _ptr(features), _ptr(pred), B,
                                            _dims(ncell)))
        return pred

    def gradients(self, features, target, ncell):
        """(loss, gradient of every parameter) without an update."""
        self._sync()
        g = np.empty(self.num_params, dtype=np.float32)
        loss = C.c_float()
        check_unet(self._L.cmi_unet_gradients(self._h, _ptr(features), _ptr(target),
                                              features.shape[0], _dims(ncell), C.byref(loss),
                                              g.ctypes.data))
        return float(loss.value), g

    def train_step(self, features, target, ncell, lr):
        self._sync()
        loss = C.c_float()
        check_unet(self._L.cmi_unet_train_step(self._h, _ptr(features), _ptr(target),
                                               features.shape[0], _dims(ncell), float(lr),
                                               C.byref(loss)))
        return float(loss.value)

    def set_loss_weight(self, over_weight):
        """Weight of the squared error where the prediction is above the target
        (x_H too high) in the training loss; 1 = mean squared error."""
        check_unet(self._L.cmi_unet_set_loss_weight(self._h, float(over_weight)))

    def features(self, nH_cube, grid, out=None, norm=None, ratio_factor=None):
        """Features [cells, 3] of one grid from its FP64 n_H (torch, device,
        cube order) and the GridSpec's box, sources and recombination rate;
        ``norm`` defaults to the network's normalisation.  ``ratio_factor`` >
        1 computes channel 2 on the grid that much coarser and interpolates it
        (default: the network's own setting, 1 unless its weights say)."""
        import torch
        self._sync()
        n = int(np.prod(grid.ncell))
        if out is None:
            out = torch.empty((n, NUM_FEATURES), dtype=torch.float32, device=nH_cube.device)
        dims = (C.c_int32 * 3)(*[int(v) for v in grid.ncell])
        box = np.ascontiguousarray(grid.box, dtype=np.float64)
        src = np.ascontiguousarray(np.asarray(grid.sources, dtype=np.float64).reshape(-1, 4))
        nm = np.ascontiguousarray(self.norm if norm is None else norm, dtype=np.float32)
        if ratio_factor is None:
            ratio_factor = self.ratio_factor
        check_unet(self._L.cmi_unet_features_coarse_ratio(
            self._h, _ptr(nH_cube), dims, box.ctypes.data, src.ctypes.data, src.shape[0],
            float(grid.recombination_rate), nm.ctypes.data, int(ratio_factor), _ptr(out)))
        return out

    @property
    def ratio_factor(self):
        meta = getattr(self, "meta", {}) or {}
        return int(meta["ratio_factor"]) if "ratio_factor" in meta else 1

    def to_neutral_fraction(self, pred, log10_min=LOG10_XH_MIN):
        import torch
        self._sync()
        x = torch.empty(pred.numel(), dtype=torch.float64, device=pred.device)
        check_unet(self._L.cmi_unet_to_neutral_fraction(self._h, _ptr(pred), _ptr(x),
                                                        pred.numel(), float(log10_min)))
        return x

    def fit_normalisation(self, nH_cubes, grids, sample=64):
        """Feature means / scales from (up to ``sample`` of) a set of grids,
        computed from the raw features on the GPU."""
        import torch
        raw = np.array([0.0, 1.0] * NUM_FEATURES, dtype=np.float32)
        acc = []
        for n, g in list(zip(nH_cubes, grids))[:sample]:
            t = torch.from_numpy(np.ascontiguousarray(n, dtype=np.float64).ravel())
            acc.append(self.features(t.to(f"cuda:{self.device}"), g, norm=raw).cpu().numpy())
        a = np.concatenate(acc)
        self.norm = np.stack([a.mean(axis=0), a.std(axis=0) + 1e-6], axis=1).ravel() \
            .astype(np.float32)


def stromgren_ratio(grid, nH_cube, nref=1e8):
    """log10 sum_i L_i / (4 pi alpha R_i) at the cell centres (cube order), R_i
    the midpoint sum of n_H^2 r^2 dr along the ray from source i in
    ceil(r / (h / 2)) steps (h the smallest cell side), n_H of the cell holding
    each sample: the features kernel's sum with the same FP32 operations, for
    tests."""
    f32 = np.float32
    box = np.asarray(grid.box, dtype=np.float64)
    n3 = tuple(int(v) for v in grid.ncell)
    cell = box[3:] / np.array(n3, dtype=np.float64)
    hmin = cell.min()
    nrel = (np.asarray(nH_cube, dtype=np.float64).reshape(n3) * (1.0 / nref)).astype(f32)
    idx = np.meshgrid(*[np.arange(n) for n in n3], indexing="ij")
    total = np.zeros(n3)
    for s in np.asarray(grid.sources, dtype=np.float64).reshape(-1, 4):
        p = [box[a] + (idx[a] + 0.5) * cell[a] for a in range(3)]
        dm = [p[a] - s[a] for a in range(3)]
        sc = [f32((s[a] - box[a]) / cell[a]) for a in range(3)]
        dc = [(dm[a] / cell[a]).astype(f32) for a in range(3)]
        r = np.sqrt((dm[0] * dm[0] + dm[1] * dm[1]) + dm[2] * dm[2])
        rh = (r / hmin).astype(f32)
        nstep = np.maximum(1, np.ceil(rh / f32(0.5)).astype(np.int64))
        inv = (f32(1.0) / nstep.astype(f32)).astype(f32)
        col = np.zeros(n3, dtype=f32)
        for k in range(int(nstep.max())):
            on = k < nstep
            t = ((f32(k) + f32(0.5)) * inv).astype(f32)
            c = [np.clip(np.floor(sc[a] + t * dc[a]).astype(np.int64), 0, n3[a] - 1)
                 for a in range(3)]
            n = nrel[c[0], c[1], c[2]]
            rr = (t * rh).astype(f32)
            col = np.where(on, (col + (n * n) * (rr * rr)).astype(f32), col)
        R = col.astype(np.float64) * (rh.astype(np.float64) * inv.astype(np.float64)) * \
            nref * nref * hmin * hmin * hmin
        total += s[3] / (4.0 * np.pi * grid.recombination_rate * np.maximum(R, 1e-300))
    return np.log10(np.clip(total, 1e-30, 1e30))


def stromgren_ratio_coarse(grid, nH_cube, factor):
    """Channel 2 as cmi_unet_features_coarse_ratio computes it, for tests: the
    ray sums of ``stromgren_ratio`` on n_H block-averaged by ``factor``, then
    trilinear interpolation in log10 (coarse cell centres at fine coordinate
    (c + 0.5) factor - 0.5, edge values held outside them)."""
    from .engine import GridSpec
    n3 = tuple(int(v) for v in grid.ncell)
    m3 = tuple(v // factor for v in n3)
    cube = np.asarray(nH_cube, dtype=np.float64).reshape(n3)
    coarse = cube.reshape(m3[0], factor, m3[1], factor, m3[2], factor).mean(axis=(1, 3, 5))
    cg = GridSpec(box=grid.box, ncell=m3, num_subgrid=(1, 1, 1),
                  recombination_rate=grid.recombination_rate,
                  cross_section=grid.cross_section, sources=list(grid.sources))
    lr = stromgren_ratio(cg, coarse).reshape(m3).astype(np.float32).astype(np.float64)
    axes = []
    for k in range(3):
        u = np.clip((np.arange(n3[k]) + 0.5) / factor - 0.5, 0.0, m3[k] - 1)
        lo = np.minimum(np.floor(u).astype(np.int64), m3[k] - 1)
        axes.append((lo, np.minimum(lo + 1, m3[k] - 1), u - lo))
    out = np.zeros(n3)
    for c in range(8):
        idx, w = [], 1.0
        for k, bit in enumerate((4, 2, 1)):
            lo, hi, t = axes[k]
            sel = hi if c & bit else lo
            wk = t if c & bit else 1.0 - t
            shape = [1, 1, 1]
            shape[k] = n3[k]
            idx.append(sel.reshape(shape))
            w = w * wk.reshape(shape)
        out += w * lr[idx[0], idx[1], idx[2]]
    return out


def flux_proxy(grid):
    """log10 sum_i L_i / (4 pi r_i^2) at the cell centres (cube order), r
    clamped to half a cell; the same quantity the features kernel computes."""
    box = np.asarray(grid.box, dtype=np.float64)
    n = tuple(int(v) for v in grid.ncell)
    cell = box[3:] / np.array(n)
    axes = [box[a] + (np.arange(n[a]) + 0.5) * cell[a] for a in range(3)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    flux = np.zeros(n)
    rmin = 0.5 * cell.min()
    for s in np.asarray(grid.sources, dtype=np.float64).reshape(-1, 4):
        r = np.maximum(np.sqrt((X - s[0]) ** 2 + (Y - s[1]) ** 2 + (Z - s[2]) ** 2), rmin)
        flux += s[3] / (4.0 * np.pi * r ** 2)
    return np.log10(np.maximum(flux, 1e-300))


# ---------------------------------------------------------------------------
# training data from the plain method
# ---------------------------------------------------------------------------
def run_configs(seeds, ncell=64, packets_per_cell=5, num_sources=4, sigma_ln=1.0):
    """Log-normal plain-method configurations (64^3 as 4^3 subgrids of 16^3)."""
    from .problems import lognormal_config
    out = []
    for s in seeds:
        g, nH = lognormal_config(ncell=ncell, num_subgrid=ncell // 16,
                                 num_photon=int(round(packets_per_cell * ncell ** 3)),
                                 num_sources=num_sources, sigma_ln=sigma_ln, seed=int(s))
        out.append((g, nH))
    return out


def generate_runs(seeds, ncell=64, packets_per_cell=5, iterations=24, average=6, batch=64,
                  device=0, log=None):
    """Plain-method runs from x_H = 1e-6, ``batch`` instances per context,
    ``iterations`` iterations each (well past convergence); the label is log10
    of x_H averaged over the last ``average`` iterations (less Monte Carlo
    noise).

    Returns (grids, nH cubes [N, n, n, n], labels log10 x_H [N, n, n, n]
    float32, dx [iterations, N]: the mean |delta x_H| of every iteration)."""
    from .engine import TransportEngine, blocked_to_cube
    grids, cubes, labels, dxs = [], [], [], []
    seeds = list(seeds)
    for b0 in range(0, len(seeds), batch):
        cfgs = run_configs(seeds[b0: b0 + batch], ncell, packets_per_cell)
        specs = [g for g, _ in cfgs]
        t0 = time.perf_counter()
        with TransportEngine(specs, precision="fp32", device=device) as eng:
            for i, (_, nH) in enumerate(cfgs):
                eng.set_fields(i, nH)
            st = eng.run_iterations(iterations - average, seed=1000 + b0)
            acc = [np.zeros(int(np.prod(g.ncell))) for g in specs]
            for k in range(average):
                st += eng.run_iterations(1, seed=5000 + b0 + k)
                for i in range(len(specs)):
                    acc[i] += eng.get_fields(i, layout="cube", intensity=False)[0]
        dxs.append(np.array([[s[i]["mean_abs_dx"] for i in range(len(specs))] for s in st]))
        for i, (g, nH) in enumerate(cfgs):
            grids.append(g)
            cubes.append(blocked_to_cube(nH, g.ncell, g.num_subgrid).astype(np.float64))
            x = np.maximum(acc[i] / average, 10.0 ** LOG10_XH_MIN)
            labels.append(np.log10(x).reshape(g.ncell).astype(np.float32))
        if log:
            log(f"runs {b0}-{b0 + len(cfgs) - 1}: {time.perf_counter() - t0:.1f} s; mean "
                f"|dx| per iteration {np.round(dxs[-1].mean(axis=1), 4).tolist()}")
    return grids, np.stack(cubes), np.stack(labels), np.concatenate(dxs, axis=1)


def iterations_to_tolerance(dx, tolerance, min_iterations=2):
    """First iteration (1-based) >= min_iterations whose mean |dx| < tolerance,
    per run (0: never), from a [iterations, runs] array."""
    ok = dx < tolerance
    ok[: min_iterations - 1] = False
    first = np.argmax(ok, axis=0) + 1
    return np.where(ok.any(axis=0), first, 0)


def build_features(net, grids, cubes):
    """Features of every run on the GPU: torch [N, cells, 3]."""
    import torch
    n = int(np.prod(grids[0].ncell))
    out = torch.empty((len(grids), n, NUM_FEATURES), dtype=torch.float32,
                      device=f"cuda:{net.device}")
    for i, (g, c) in enumerate(zip(grids, cubes)):
        nH = torch.from_numpy(np.ascontiguousarray(c).ravel()).to(out.device)
        net.features(nH, g, out=out[i])
    return out


def train(net, feats, labels, ncell, epochs=10, batch=8, lr=2e-3, lr_final=2e-4, seed=0,
          log=None):
    """Adam over shuffled mini-batches, learning rate decaying geometrically
    from lr to lr_final.  feats [N, cells, 2], labels [N, cells] (torch)."""
    import torch
    N = feats.shape[0]
    rng = np.random.default_rng(seed)
    steps = epochs * (N // batch)
    history = []
    k = 0
    t0 = time.perf_counter()
    for ep in range(epochs):
        order = rng.permutation(N)
        losses = []
        for b in range(N // batch):
            idx = torch.from_numpy(order[b * batch:(b + 1) * batch]).to(feats.device)
            f = feats.index_select(0, idx).contiguous()
            t = labels.index_select(0, idx).contiguous()
            rate = lr * (lr_final / lr) ** (k / max(1, steps - 1))
            losses.append(net.train_step(f, t, ncell, rate))
            k += 1
        history.append(float(np.mean(losses)))
        if log:
            log(f"epoch {ep}: loss {history[-1]:.5f} ({time.perf_counter() - t0:.1f} s)")
    return history


def generate_large_runs(net, seeds, iterations=24, average=6, ratio_factor=4, device=0,
                        log=None, num_photon=100_000_000):
    """Runs of the large generator (256^3 as 16^3 subgrids of 16^3, sigma_ln =
    1.5, 16 sources; problems.large_config) with ``num_photon`` packets per
    iteration, kept on the device: raw features [N, cells, 3] (channel 2 from
    the grid coarser by ``ratio_factor``) and labels log10 x_H [N, cells] of the
    long plain run (``iterations`` from x_H = 1e-6, the last ``average``
    averaged)."""
    import torch
    from .engine import blocked_to_cube
    from .problems import large_config
    raw = np.array([0.0, 1.0] * NUM_FEATURES, dtype=np.float32)
    feats, labels, grids = None, None, []
    t0 = time.perf_counter()
    for i, sd in enumerate(seeds):
        g, nH = large_config(seed=int(sd), num_photon=int(num_photon))
        ncell = int(np.prod(g.ncell))
        if feats is None:
            feats = torch.empty((len(seeds), ncell, NUM_FEATURES), dtype=torch.float32,
                                device=f"cuda:{device}")
            labels = torch.empty((len(seeds), ncell), dtype=torch.float32, device=feats.device)
        x = reference_field(g, nH, iterations=iterations, average=average, seed=7000 + i,
                            device=device)
        labels[i] = torch.from_numpy(np.log10(np.maximum(x, 10.0 ** LOG10_XH_MIN))
                                     .astype(np.float32)).to(feats.device)
        cube = torch.from_numpy(blocked_to_cube(nH, g.ncell, g.num_subgrid)).to(feats.device)
        net.features(cube, g, out=feats[i], norm=raw, ratio_factor=ratio_factor)
        grids.append(g)
        if log and (i % 8 == 7 or i == len(seeds) - 1):
            log(f"large runs {i + 1}/{len(seeds)}: {time.perf_counter() - t0:.1f} s")
    return grids, feats, labels


def random_crops(feats, labels, ncell, crop, batch, rng):
    """``batch`` random crop^3 windows of random runs: features [batch, crop^3,
    3] and labels [batch, crop^3], contiguous (the network's zero padding sees
    the window edge; the features already carry the whole grid's sources)."""
    import torch
    n0, n1, n2 = ncell
    f = feats.view(feats.shape[0], n0, n1, n2, NUM_FEATURES)
    t = labels.view(labels.shape[0], n0, n1, n2)
    fo, to = [], []
    for _ in range(batch):
        r = int(rng.integers(feats.shape[0]))
        z, y, x = (int(rng.integers(n - crop + 1)) for n in ncell)
        fo.append(f[r, z:z + crop, y:y + crop, x:x + crop])
        to.append(t[r, z:z + crop, y:y + crop, x:x + crop])
    return (torch.stack(fo).reshape(batch, -1, NUM_FEATURES).contiguous(),
            torch.stack(to).reshape(batch, -1).contiguous())


def train_crops(net, feats, labels, ncell, steps=3000, crop=64, batch=8, lr=1e-3,
                lr_final=1e-4, seed=0, log=None):
    """Adam on random crop^3 windows of the large runs (normalised features),
    learning rate decaying geometrically from lr to lr_final."""
    rng = np.random.default_rng(seed)
    hist, acc = [], []
    t0 = time.perf_counter()
    for k in range(steps):
        f, t = random_crops(feats, labels, ncell, crop, batch, rng)
        rate = lr * (lr_final / lr) ** (k / max(1, steps - 1))
        acc.append(net.train_step(f, t, (crop,) * 3, rate))
        if (k + 1) % 250 == 0:
            hist.append(float(np.mean(acc)))
            acc = []
            if log:
                log(f"step {k + 1}: loss {hist[-1]:.5f} ({time.perf_counter() - t0:.1f} s)")
    return hist


def normalise_features(feats, norm):
    """In place: (raw - norm[2k]) / norm[2k + 1] per channel."""
    for k in range(NUM_FEATURES):
        feats[..., k].sub_(float(norm[2 * k])).div_(float(norm[2 * k + 1]))


def evaluate_loss(net, feats, labels, ncell, batch=8):
    import torch
    tot, n = 0.0, 0
    with torch.no_grad():
        for b in range(0, feats.shape[0], batch):
            f = feats[b: b + batch].contiguous()
            p = net.forward(f, ncell)
            tot += float(((p - labels[b: b + batch]) ** 2).sum())
            n += p.numel()
    return tot / n


# ---------------------------------------------------------------------------
# warm start and the convergence comparison
# ---------------------------------------------------------------------------
def training_ncell(net):
    """Cells per axis of the grids the network was trained on (64 unless its
    weights say otherwise)."""
    meta = getattr(net, "meta", {}) or {}
    return int(meta["ncell"]) if "ncell" in meta else 64


def predict_log_xH(net, grid, nH_dev):
    """log10 x_H predicted for ``grid`` (torch FP32, cube order).

    A grid finer than the training grid by an integer factor per axis is
    predicted at the training resolution: n_H is block-averaged to it (the
    sources keep their positions), the network runs there and its prediction is
    upsampled back (nearest neighbour).  The features and the receptive field
    are then the ones the network was trained on; the plain iterations that
    follow resolve the finer structure."""
    import torch
    from .engine import GridSpec
    n = tuple(int(v) for v in grid.ncell)
    base = training_ncell(net)
    f = n[0] // base if n[0] % base == 0 else 1
    if f > 1 and all(v == base * f for v in n):
        coarse = GridSpec(box=grid.box, ncell=(base,) * 3, num_subgrid=(1, 1, 1),
                          recombination_rate=grid.recombination_rate,
                          cross_section=grid.cross_section, sources=list(grid.sources))
        nc = torch.empty(base ** 3, dtype=torch.float64, device=nH_dev.device)
        net._sync()
        check_unet(net._L.cmi_unet_block_mean(net._h, _ptr(nH_dev), (C.c_int32 * 3)(*n), f,
                                              _ptr(nc)))
        feats = net.features(nc, coarse).unsqueeze(0).contiguous()
        pc = net.forward(feats, coarse.ncell)
        out = torch.empty(int(np.prod(n)), dtype=torch.float32, device=nH_dev.device)
        check_unet(net._L.cmi_unet_upsample_nearest(net._h, _ptr(pc), (C.c_int32 * 3)(*(base,) * 3),
                                                    f, _ptr(out)))
        return out
    feats = net.features(nH_dev, grid).unsqueeze(0).contiguous()
    return net.forward(feats, grid.ncell).reshape(-1)


def warm_start(net, engine, instance, nH_cube, log10_min=LOG10_XH_MIN):
    """Predict x_H for an engine instance and load it.  ``nH_cube``: n_H in
    cube order, a torch CUDA tensor (FP64) or a host array (copied first)."""
    import torch
    grid = engine.grids[instance]
    dev = f"cuda:{net.device}"
    if isinstance(nH_cube, torch.Tensor):
        nH = nH_cube.reshape(-1)
    else:
        nH = torch.from_numpy(np.ascontiguousarray(nH_cube, dtype=np.float64).ravel()).to(dev)
    pred = predict_log_xH(net, grid, nH)
    x = net.to_neutral_fraction(pred, log10_min)
    torch.cuda.synchronize(dev)
    engine.set_fields_device(instance, 0, x.data_ptr(), layout="cube")
    return x


def warm_breakdown(net, engine, instance, nH_dev, repeats=5):
    """Milliseconds of the warm start's stages (prediction: features and
    network, at the training resolution for finer grids; x_H into the engine),
    each bracketed by device synchronisations."""
    import torch
    grid = engine.grids[instance]
    t = {"predict": 0.0, "load": 0.0}
    for _ in range(repeats):
        torch.cuda.synchronize(net.device)
        t0 = time.perf_counter()
        pred = predict_log_xH(net, grid, nH_dev)
        torch.cuda.synchronize(net.device)
        t1 = time.perf_counter()
        x = net.to_neutral_fraction(pred)
        engine.set_fields_device(instance, 0, x.data_ptr(), layout="cube")
        t2 = time.perf_counter()
        t["predict"] += (t1 - t0) * 1e3 / repeats
        t["load"] += (t2 - t1) * 1e3 / repeats
    return t


def reference_field(grid, nH_blocked, iterations=24, average=6, seed=5000, device=0):
    """x_H (cube order) of a long plain run: ``iterations`` from x_H = 1e-6,
    averaged over the last ``average`` (the converged answer, less noise)."""
    from .engine import TransportEngine
    with TransportEngine(grid, precision="fp32", device=device) as eng:
        eng.set_fields(0, nH_blocked, np.full(nH_blocked.size, 1e-6))
        eng.run_iterations(iterations - average, seed=seed)
        acc = np.zeros(int(np.prod(grid.ncell)))
        for k in range(average):
            eng.run_iterations(1, seed=seed + 1 + k)
            acc += eng.get_fields(0, layout="cube", intensity=False)[0]
    return acc / average


def time_to_converge(net, grid, nH_blocked, x_reference=None, tolerance=0.01,
                     max_iterations=60, seed=7, device=0, plain_spread=True):
    """Iterations and wall time (s) to convergence (mean |delta x_H| <
    tolerance, cmi_run_until_converged) from x_H = 1e-6 and from the warm
    start, same grid and packet seed.  Wall time covers the features, the
    network and the iterations, with n_H already on the device and both paths
    warmed up (graph capture, network buffers).  With ``x_reference`` (cube
    order) also the mean |x - x_reference| of each converged field; always the
    mean |x_plain - x_warm|."""
    import torch
    from .engine import TransportEngine, blocked_to_cube
    cube = blocked_to_cube(nH_blocked, grid.ncell, grid.num_subgrid)
    # n_H is resident on the device, like the engine's copy
    cube_dev = torch.from_numpy(np.ascontiguousarray(cube).ravel()).to(f"cuda:{device}")
    out = {}
    fields = {}
    for mode in ("plain", "warm"):
        with TransportEngine(grid, precision="fp32", device=device) as eng:
            eng.set_fields(0, nH_blocked, np.full(nH_blocked.size, 1e-6))
            eng.run_iterations(1, seed=99)  # warm-up: graph capture, first touch
            if mode == "warm":
                warm_start(net, eng, 0, cube_dev)  # warm-up of the network path
                out["warm_breakdown_ms"] = warm_breakdown(net, eng, 0, cube_dev)
            eng.set_fields(0, None, np.full(nH_blocked.size, 1e-6))
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            if mode == "warm":
                warm_start(net, eng, 0, cube_dev)
            stats, at = eng.run_until_converged(tolerance, max_iterations=max_iterations,
                                                min_iterations=2, seed=seed)
            eng.synchronize()
            dt = time.perf_counter() - t0
            fields[mode] = eng.get_fields(0, layout="cube", intensity=False)[0]
            out[mode] = {"iterations": int(at[0]) or len(stats), "converged": bool(at[0]),
                         "seconds": dt,
                         "dx": [round(s[0]["mean_abs_dx"], 5) for s in stats]}
            if x_reference is not None:
                out[mode]["error_vs_reference"] = float(
                    np.mean(np.abs(fields[mode] - np.ravel(x_reference))))
    out["mean_abs_dx_between"] = float(np.mean(np.abs(fields["plain"] - fields["warm"])))
    out["speedup"] = out["plain"]["seconds"] / out["warm"]["seconds"]
    if plain_spread:
        # the same plain run with other packets: the Monte Carlo spread that
        # any two converged fields show
        with TransportEngine(grid, precision="fp32", device=device) as eng:
            eng.set_fields(0, nH_blocked, np.full(nH_blocked.size, 1e-6))
            eng.run_until_converged(tolerance, max_iterations=max_iterations, min_iterations=2,
                                    seed=seed + 1)
            x2 = eng.get_fields(0, layout="cube", intensity=False)[0]
        out["mean_abs_dx_plain_vs_plain"] = float(np.mean(np.abs(fields["plain"] - x2)))
    return out


def time_steps(steps, batch=8, ncell=64, log=print, warmup=3):
    """Wall time per training step and per inference pass of the default
    network on synthetic features (device-synchronised, after warm-up)."""
    import json

    import torch
    rng = np.random.default_rng(0)
    n = ncell ** 3
    f = torch.from_numpy(rng.normal(size=(batch, n, NUM_FEATURES)).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.normal(-1, 1, size=(batch, n)).astype(np.float32)).cuda()
    dims = (ncell,) * 3
    with UNet() as net:
        for _ in range(warmup):
            net.train_step(f, t, dims, 1e-4)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            net.train_step(f, t, dims, 1e-4)
        torch.cuda.synchronize()
        train_ms = (time.perf_counter() - t0) * 1e3 / steps
        f1 = f[:1].contiguous()
        for _ in range(warmup):
            net.forward(f1, dims)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            net.forward(f1, dims)
        torch.cuda.synchronize()
        infer_ms = (time.perf_counter() - t0) * 1e3 / steps
    log(json.dumps({"train_step_ms": train_ms, "batch": batch, "ncell": ncell,
                    "voxels_per_s": batch * n / (train_ms / 1e3),
                    "inference_ms_batch1": infer_ms}))
    return 0


def train_large(runs, steps, over_weight, out, log, ratio_factor=4, crop=64, batch=8,
                label_iterations=16, label_average=4):
    """The 256^3 weights: ``runs`` long plain runs of large_config (seeds
    300000 + i, the last sixth held out), features with channel 2 from the
    grid coarser by ``ratio_factor``, the 64^3 weights (and normalisation)
    fine-tuned on random crop^3 windows under the asymmetric loss."""
    ntrain = runs - max(1, runs // 6)
    seeds = [300_000 + i for i in range(runs)]
    net = UNet.load(DEFAULT_WEIGHTS)
    grids, feats, labels = generate_large_runs(net, seeds, iterations=label_iterations,
                                               average=label_average,
                                               ratio_factor=ratio_factor, log=log)
    normalise_features(feats, net.norm)
    ncell = grids[0].ncell
    base = float(((labels[ntrain:] - labels[:ntrain].mean(0)) ** 2).mean())
    net.set_loss_weight(over_weight)
    hist = train_crops(net, feats[:ntrain], labels[:ntrain], ncell, steps=steps, crop=crop,
                       batch=batch, log=log)
    net.set_loss_weight(1.0)
    val = evaluate_loss(net, feats[ntrain:], labels[ntrain:], ncell, batch=1)
    log(f"held-out MSE {val:.4f} (mean-field baseline {base:.4f})")
    net.save(out, ncell=int(ncell[0]), ratio_factor=ratio_factor, val_mse=val,
             baseline_mse=base, over_weight=over_weight, train_loss=np.array(hist),
             generator="large_config: 256^3, sigma_ln=1.5, 16 sources, 1e8 packets",
             train_seeds=np.array([seeds[0], seeds[ntrain]]),
             val_seeds=np.array([seeds[ntrain], seeds[-1] + 1]), steps=steps, crop=crop,
             batch=batch, label_iterations=label_iterations, label_average=label_average,
             init=os.path.basename(DEFAULT_WEIGHTS), lr=np.array([1e-3, 1e-4]))
    return 0


def main(argv=None):
    import argparse
    import json

    import torch
    ap = argparse.ArgumentParser(description="train the warm-start U-Net on plain-method runs")
    ap.add_argument("--runs", type=int, default=2000)
    ap.add_argument("--ncell", type=int, default=64)
    ap.add_argument("--packets-per-cell", type=float, default=5)
    ap.add_argument("--label-iterations", type=int, default=24)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--tolerance", type=float, default=0.01)
    ap.add_argument("--eval", type=int, default=16, help="held-out runs for the wall-time test")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--report", default=None)
    ap.add_argument("--time-steps", type=int, default=0,
                    help="only time this many training steps and inference passes on "
                         "synthetic 64^3 data (batch --batch) and exit")
    ap.add_argument("--large", action="store_true",
                    help="fine-tune the 64^3 weights on the 256^3 generator instead "
                         "(--runs long runs, 1/6 held out; writes the 256^3 weights)")
    ap.add_argument("--steps", type=int, default=6000, help="--large: training steps")
    ap.add_argument("--over-weight", type=float, default=16.0,
                    help="--large: loss weight of predictions above the target")
    a = ap.parse_args(argv)
    log = (lambda s: print(s, flush=True))
    torch.cuda.set_device(0)
    if a.time_steps:
        return time_steps(a.time_steps, a.batch, a.ncell, log)
    if a.large:
        return train_large(a.runs, a.steps, a.over_weight,
                           LARGE_WEIGHTS if a.out == DEFAULT_WEIGHTS else a.out, log)
    ntrain = int(round(0.8 * a.runs))
    seeds = [100_000 + i for i in range(a.runs)]
    t0 = time.perf_counter()
    grids, cubes, labels, dx = generate_runs(seeds, ncell=a.ncell,
                                             packets_per_cell=a.packets_per_cell,
                                             iterations=a.label_iterations, log=log)
    t_gen = time.perf_counter() - t0
    plain_its = iterations_to_tolerance(dx, a.tolerance)
    log(f"plain method: iterations to mean |dx| < {a.tolerance}: mean {plain_its.mean():.2f}, "
        f"not reached {int(np.sum(plain_its == 0))}; noise floor (last iterations) "
        f"{dx[-4:].mean():.4f}")
    net = UNet()
    net.fit_normalisation(cubes[:ntrain], grids[:ntrain])
    feats = build_features(net, grids, cubes)
    lab = torch.from_numpy(labels.reshape(len(grids), -1)).to(feats.device)
    ncell = grids[0].ncell
    t0 = time.perf_counter()
    hist = train(net, feats[:ntrain], lab[:ntrain], ncell, epochs=a.epochs, batch=a.batch,
                 lr=a.lr, log=log)
    t_train = time.perf_counter() - t0
    val = evaluate_loss(net, feats[ntrain:], lab[ntrain:], ncell)
    base = float(((lab[ntrain:] - lab[:ntrain].mean(0)) ** 2).mean())
    log(f"held-out MSE {val:.5f} (mean-field baseline {base:.5f})")
    net.save(a.out, train_loss=np.array(hist), val_mse=val, baseline_mse=base,
             runs=a.runs, ncell=a.ncell, tolerance=a.tolerance,
             packets_per_cell=a.packets_per_cell)
    ev = []
    for i in range(ntrain, min(ntrain + a.eval, a.runs)):
        g, nH = run_configs([seeds[i]], a.ncell, a.packets_per_cell)[0]
        ev.append(time_to_converge(net, g, nH, x_reference=10.0 ** labels[i].astype(np.float64),
                                   tolerance=a.tolerance))
        log(json.dumps(ev[-1]))

    def mean(key, sub):
        return float(np.mean([e[key][sub] for e in ev]))
    rep = {"runs": a.runs, "train": ntrain, "generation_s": t_gen, "training_s": t_train,
           "train_loss": hist, "val_mse": val, "baseline_mse": base,
           "tolerance": a.tolerance, "noise_floor_dx": float(dx[-4:].mean()),
           "plain_iterations_mean": mean("plain", "iterations"),
           "warm_iterations_mean": mean("warm", "iterations"),
           "plain_seconds_mean": mean("plain", "seconds"),
           "warm_seconds_mean": mean("warm", "seconds"),
           "speedup_median": float(np.median([e["speedup"] for e in ev])),
           "plain_error_vs_reference": mean("plain", "error_vs_reference"),
           "warm_error_vs_reference": mean("warm", "error_vs_reference"),
           "mean_abs_dx_between_mean": float(np.mean([e["mean_abs_dx_between"] for e in ev])),
           "mean_abs_dx_plain_vs_plain_mean": float(np.mean(
               [e["mean_abs_dx_plain_vs_plain"] for e in ev])),
           "eval": ev}
    if a.report:
        with open(a.report, "w") as f:
            json.dump(rep, f, indent=1)
    log(json.dumps({k: v for k, v in rep.items() if k not in ("eval", "train_loss")}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
