"""Synthetic inputs of the benchmark configurations (seeded, no external data).

* ``stromgren``      -- the reference's own test: uniform n_H = 1e8 m^-3, one
  source of 4.26e49 s^-1 at the centre of a +-5 pc box (params_single_uniform.txt,
  testDensitySubGrid_omp.cpp:2001-2015).
* ``lognormal_density`` -- ln n = mu + s * g, g unit-variance Gaussian white
  noise smoothed by a Gaussian kernel (periodic FFT) and renormalised;
  mu = ln(mean) - s^2 / 2 so that <n> = mean.
* ``random_sources`` -- positions uniform in the box, luminosities
  log-uniform between two bounds.
* ``lognormal_config`` / ``batch_configs`` / ``large_config`` -- the log-normal
  plain-method workload, the batched set of uneven instances and the large
  256^3 run.
* ``stromgren_profile`` -- the semi-analytic neutral-fraction profile and
  Stromgren radius of scripts/plot_neutral_fraction_profile.py:60-82.
* ``reference_setup`` -- the reference driver's own initial conditions for a
  params.txt (its random density field and random sources included), drawn
  from the host generator seeded as the driver seeds it.
"""
from __future__ import annotations

import numpy as np

from .engine import PARSEC, GridSpec, cube_to_blocked

BOX_10PC = (-5.0 * PARSEC, -5.0 * PARSEC, -5.0 * PARSEC, 10.0 * PARSEC, 10.0 * PARSEC,
            10.0 * PARSEC)


def stromgren(ncell=64, num_subgrid=8, num_photon=1_000_000, alpha=4.0e-19,
              luminosity=4.26e49):
    g = GridSpec(box=BOX_10PC, ncell=(ncell,) * 3, num_subgrid=(num_subgrid,) * 3,
                 recombination_rate=alpha, sources=[(0.0, 0.0, 0.0, luminosity)],
                 num_photon=num_photon)
    nH = np.full(g.num_cells, 1.0e8)
    return g, nH


def lognormal_density(ncell, sigma_ln=1.0, smoothing_cells=4.0, mean=1.0e8, seed=42):
    """Cube (nx, ny, nz) of a log-normal number density field."""
    rng = np.random.default_rng(seed)
    n = tuple(int(v) for v in (ncell if np.ndim(ncell) else (ncell,) * 3))
    g = rng.standard_normal(n)
    k = [np.fft.fftfreq(m) for m in n]
    kx, ky, kz = np.meshgrid(*k, indexing="ij")
    kern = np.exp(-0.5 * (2 * np.pi) ** 2 * smoothing_cells ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    gs = np.fft.ifftn(np.fft.fftn(g) * kern).real
    gs = (gs - gs.mean()) / gs.std()
    mu = np.log(mean) - 0.5 * sigma_ln ** 2
    return np.exp(mu + sigma_ln * gs)


def random_sources(box, count, log_lum=(48.0, 49.0), seed=43):
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=np.float64)
    pos = box[:3] + rng.uniform(size=(count, 3)) * box[3:]
    lum = 10.0 ** rng.uniform(log_lum[0], log_lum[1], size=count)
    return [tuple(p) + (float(l),) for p, l in zip(pos, lum)]


def lognormal_config(ncell=128, num_subgrid=8, num_photon=10_000_000, num_sources=4,
                     sigma_ln=1.0, seed=42, alpha=4.0e-19):
    """Log-normal plain-method workload (128^3 as 8^3 subgrids of 16^3 by default).

    Returns (GridSpec, n_H in subgrid-blocked order)."""
    g = GridSpec(box=BOX_10PC, ncell=(ncell,) * 3, num_subgrid=(num_subgrid,) * 3,
                 recombination_rate=alpha, num_photon=num_photon)
    g.sources = random_sources(g.box, num_sources, seed=seed + 1)
    cube = lognormal_density(ncell, sigma_ln=sigma_ln, seed=seed)
    return g, cube_to_blocked(cube, g.ncell, g.num_subgrid)


def batch_configs(count=64, sides=(32, 48, 64, 96, 128), sigma_range=(0.5, 1.5),
                  max_sources=4, packets_per_cell=5, sub_cells=16, seed=7, alpha=4.0e-19,
                  select=None):
    """Independent instances of uneven size, density contrast and source count.

    Returns a list of (GridSpec, n_H blocked); with ``select`` (a set of
    indices) the density of the other instances is None (not generated)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        side = int(rng.choice(sides))
        sc = sub_cells if side % sub_cells == 0 else 8
        s_ln = float(rng.uniform(*sigma_range))
        nsrc = int(rng.integers(1, max_sources + 1))
        g = GridSpec(box=BOX_10PC, ncell=(side,) * 3, num_subgrid=(side // sc,) * 3,
                     recombination_rate=alpha, num_photon=packets_per_cell * side ** 3)
        g.sources = random_sources(g.box, nsrc, seed=seed * 1000 + i)
        if select is not None and i not in select:
            out.append((g, None))
            continue
        cube = lognormal_density(side, sigma_ln=s_ln, seed=seed * 1000 + i)
        out.append((g, cube_to_blocked(cube, g.ncell, g.num_subgrid)))
    return out


def large_config(ncell=256, num_subgrid=16, num_photon=100_000_000, num_sources=16,
                 sigma_ln=1.5, seed=42, alpha=4.0e-19):
    """The large log-normal run: 256^3 as 16^3 subgrids of 16^3, sigma_ln = 1.5,
    16 sources, 1e8 packets per iteration."""
    return lognormal_config(ncell=ncell, num_subgrid=num_subgrid, num_photon=num_photon,
                            num_sources=num_sources, sigma_ln=sigma_ln, seed=seed, alpha=alpha)


def dust_sphere(ncell=32, num_subgrid=4):
    """The dust driver's test medium (testDensitySubGrid_omp_dust.cpp:2073-2091):
    box [-1, 1]^3 (m), n_H = 1 in cells whose midpoint lies within radius 1,
    0 outside; x_H = 1 (the state after the driver's first balance, whose J
    is 0).  Returns (GridSpec, n_H blocked, x_H blocked)."""
    from .outputs import cell_centres_blocked
    g = GridSpec(box=(-1.0, -1.0, -1.0, 2.0, 2.0, 2.0), ncell=(ncell,) * 3,
                 num_subgrid=(num_subgrid,) * 3)
    pos = cell_centres_blocked(g)
    r = np.sqrt((pos * pos).sum(axis=1))
    nH = np.where(r < 1.0, 1.0, 0.0)
    return g, nH, np.ones_like(nH)


def stromgren_profile(alpha=4.0e-19, nH=1.0e8, Q=4.26e49, sigma=6.3e-22,
                      reemission_probability=0.0, samples=1200):
    """Semi-analytic x_H(r) and R_S (scripts/plot_neutral_fraction_profile.py:60-82)."""
    Rs = (0.75 * Q / (1.0 - reemission_probability) / (np.pi * nH ** 2 * alpha)) ** (1.0 / 3.0)
    r = np.linspace(0.0, 1.2 * Rs, samples)
    x = np.zeros(r.shape)
    integral = 0.0
    factor = 0.125 * Q * sigma / (np.pi * nH * alpha)
    intfac = 0.0005 * Rs * nH * sigma
    for i in range(1, len(r)):
        A = factor * np.exp(-integral) / r[i] ** 2
        x[i] = 1.0 + A - np.sqrt(2.0 * A + A ** 2)
        integral += intfac * (x[i - 1] + x[i])
    return r, x, Rs


def cell_radii(grid: GridSpec, centre=(0.0, 0.0, 0.0)):
    """Distance of every cell centre (cube order) from `centre`."""
    box = np.asarray(grid.box)
    axes = [box[a] + (np.arange(grid.ncell[a]) + 0.5) * box[3 + a] / grid.ncell[a] - centre[a]
            for a in range(3)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    return np.sqrt(X ** 2 + Y ** 2 + Z ** 2)


def ionized_radius(xH_cube, grid: GridSpec):
    """Radius of the sphere whose volume equals the ionized volume sum(1 - x_H) dV."""
    dv = np.prod(np.asarray(grid.box[3:]) / np.asarray(grid.ncell))
    vol = float(np.sum(1.0 - np.asarray(xH_cube)) * dv)
    return (3.0 * vol / (4.0 * np.pi)) ** (1.0 / 3.0)


def reference_setup(params, threads=1):
    """The reference driver's initial conditions for ``params`` (a
    ``Parameters``), as its run with ``-t threads`` sets them up
    (testDensitySubGrid_omp.cpp:1786-2016).  Returns (GridSpec, n_H blocked).

    The host generator is RandomGenerator(42 + threads) (:1786-1790).
    * ``random_density``: 10 cosine modes, per mode four uniforms for the wave
      vector (Box-Muller pairs scaled by 4 pi / box side) and three phases;
      n_H at a cell midpoint is the mean over the modes of
      1e8 (cos(k_x x + p_x) cos(k_y y + p_y) cos(k_z z + p_z) + 1) (:1880-1934).
      Otherwise n_H = 1e8 m^-3 everywhere (the subgrid constructor's value).
    * ``number_of_sources`` > 1: positions uniform in the box (three draws
      per source, after the density's) with 4.26e48 s^-1 each; else one
      source of 4.26e49 s^-1 at the origin (:1944-2016).
    The arithmetic is the driver's, operation for operation, with the host
    libm's cos, sin and log (math module), so on the same host the field
    equals the reference's bit for bit; it takes about 1.5 s per 2^18 cells
    (one core).
    """
    import math

    from .outputs import cell_centres_blocked
    from .ranlxd import Ranlxd
    box = tuple(float(v) for v in params.box)
    rng = Ranlxd(42 + int(threads))
    g = GridSpec(box=box, ncell=tuple(int(v) for v in params.ncell),
                 num_subgrid=tuple(int(v) for v in params.num_subgrid),
                 num_photon=int(params.num_photon),
                 reemission_probability=float(params.reemission_probability))
    if params.random_density:
        modes = []
        for _ in range(10):
            u = [rng.uniform() for _ in range(4)]
            kx = math.sqrt(-2. * math.log(u[0])) * math.cos(2. * math.pi * u[1])
            ky = math.sqrt(-2. * math.log(u[0])) * math.sin(2. * math.pi * u[1])
            kz = math.sqrt(-2. * math.log(u[2])) * math.cos(2. * math.pi * u[3])
            k = (4. * math.pi * kx / box[3], 4. * math.pi * ky / box[4],
                 4. * math.pi * kz / box[5])
            phase = tuple(2. * math.pi * rng.uniform() for _ in range(3))
            modes.append((k, phase))
        mid = cell_centres_blocked(g)
        cos = np.frompyfunc(math.cos, 1, 1)  # the host libm, element by element
        nH = np.zeros(g.num_cells)
        for k, phase in modes:
            c = [cos(k[a] * mid[:, a] + phase[a]).astype(np.float64) for a in range(3)]
            nH += 1.e8 * (c[0] * c[1] * c[2] + 1.)
        nH /= 10.
    else:
        nH = np.full(g.num_cells, 1.e8)
    if params.number_of_sources > 1:
        sources = []
        for _ in range(int(params.number_of_sources)):
            pos = [box[a] + rng.uniform() * box[3 + a] for a in range(3)]
            sources.append((pos[0], pos[1], pos[2], 4.26e48))
    else:
        sources = [(0.0, 0.0, 0.0, 4.26e49)]
    g.sources = sources
    return g, nH
