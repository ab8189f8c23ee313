"""Result files in the reference's formats, from the engine's fields.

The reference driver writes the final neutral fractions at the end of a run
(testDensitySubGrid_omp.cpp:2463-2491), each format behind a compile switch:

* ``neutral_fractions.bin`` (BIN_FILE; output_neutral_fractions_binary,
  testDensitySubGrid_omp.cpp:507-521): x_H as FP64, subgrid after subgrid in
  subgrid index order, the cells of a subgrid in their own index order (ix
  slowest, iz fastest) -- the engine's "blocked" layout.
* ``neutral_fractions.dat`` (MM_FILE; output_neutral_fractions,
  testDensitySubGrid_omp.cpp:394-442, through DensitySubGrid::
  output_intensities(offset, MemoryMap&), DensitySubGrid.hpp:1738-1788): the
  same order, 60 bytes per cell -- the cell centre x, y, z, x_H and n_H as
  FP64, then five 4-byte slots for the hydro primitives, zero in the
  photoionization-only build (NO_HYDRO, testDensitySubGrid_omp.cpp:95).
  The centre is anchor + (i + 0.5) * cell_size with the subgrid's anchor =
  box anchor + index * (box side / num_subgrid) and cell_size = subgrid side
  / subgrid cells, the reference's arithmetic (testDensitySubGrid_omp.cpp:
  1826-1832, DensitySubGrid.hpp:517-519).
* HDF5 (``/PartType0/NeutralFractionH``, testDensitySubGrid_omp.cpp:453-495)
  needs libhdf5, which is not installed here: not written.

The reference's NO_HYDRO branch writes each zero slot as an 8-byte double at
4-byte steps, so every cell record spills 4 zero bytes into the next one.
Inside a subgrid the next record overwrites them; after the last cell of a
subgrid they land on the first 4 bytes (the low half of the first centre's x)
of the next subgrid's block, which corrupts that value when the next block
was written first (several threads), and past the end of the file for the
last subgrid.  The files written here have no such spill: they equal the
reference's single-thread output byte for byte.
"""
from __future__ import annotations

import numpy as np

DAT_RECORD = np.dtype([("pos", "<f8", (3,)), ("xH", "<f8"), ("nH", "<f8"),
                       ("hydro", "<f4", (5,))])
assert DAT_RECORD.itemsize == 60


def _geometry(grid):
    box = np.asarray(grid.box, dtype=np.float64)
    ncell = np.asarray(grid.ncell, dtype=np.int64)
    ns = np.asarray(grid.num_subgrid, dtype=np.int64)
    if np.any(ncell % ns):
        raise ValueError("grid cells must be a multiple of the subgrids per axis")
    sub_side = box[3:] / ns.astype(np.float64)
    sub_n = ncell // ns
    cell = sub_side / sub_n.astype(np.float64)
    return box, ns, sub_side, sub_n, cell


def cell_centres_blocked(grid):
    """[cells, 3] FP64 centres in the blocked (output) order, computed as the
    reference computes them for its result files."""
    box, ns, sub_side, sub_n, cell = _geometry(grid)
    out = np.empty((int(np.prod(ns)), int(np.prod(sub_n)), 3), dtype=np.float64)
    s = np.arange(int(np.prod(ns)))
    sidx = np.stack([s // (ns[1] * ns[2]), (s // ns[2]) % ns[1], s % ns[2]], axis=1)
    c = np.arange(int(np.prod(sub_n)))
    cidx = np.stack([c // (sub_n[1] * sub_n[2]), (c // sub_n[2]) % sub_n[1], c % sub_n[2]],
                    axis=1)
    for a in range(3):
        anchor = box[a] + sidx[:, a].astype(np.float64) * sub_side[a]          # [S]
        off = (cidx[:, a].astype(np.float64) + 0.5) * cell[a]                  # [C]
        out[:, :, a] = anchor[:, None] + off[None, :]
    return out.reshape(-1, 3)


def neutral_fractions_dat(grid, xH_blocked, nH_blocked):
    """The bytes of neutral_fractions.dat (structured array of DAT_RECORD)."""
    n = int(np.prod(grid.ncell))
    x = np.asarray(xH_blocked, dtype=np.float64).reshape(-1)
    nh = np.asarray(nH_blocked, dtype=np.float64).reshape(-1)
    if x.size != n or nh.size != n:
        raise ValueError("field size does not match the grid")
    rec = np.zeros(n, dtype=DAT_RECORD)
    rec["pos"] = cell_centres_blocked(grid)
    rec["xH"] = x
    rec["nH"] = nh
    return rec


def write_neutral_fractions_dat(path, grid, xH_blocked, nH_blocked):
    rec = neutral_fractions_dat(grid, xH_blocked, nH_blocked)
    rec.tofile(path)
    return rec.nbytes


def write_neutral_fractions_binary(path, grid, xH_blocked):
    x = np.ascontiguousarray(xH_blocked, dtype="<f8").reshape(-1)
    if x.size != int(np.prod(grid.ncell)):
        raise ValueError("field size does not match the grid")
    x.tofile(path)
    return x.nbytes


def read_neutral_fractions_dat(path):
    """Records of a neutral_fractions.dat (ours or the reference's)."""
    raw = np.fromfile(path, dtype=np.uint8)
    if raw.size % DAT_RECORD.itemsize:
        raise ValueError(f"{path}: size is not a multiple of {DAT_RECORD.itemsize} bytes")
    return raw.view(DAT_RECORD)


def read_neutral_fractions_binary(path):
    return np.fromfile(path, dtype="<f8")


def write_outputs(engine, instance, prefix="neutral_fractions", formats=("dat", "bin"),
                  nH_blocked=None):
    """Write an engine instance's x_H in the reference's formats:
    ``<prefix>.dat`` and/or ``<prefix>.bin``.  The .dat file also carries n_H:
    pass the blocked n_H given to the engine (the engine keeps it only on the
    device).  Returns {format: path}."""
    grid = engine.grids[instance]
    x, _ = engine.get_fields(instance, layout="blocked", intensity=False)
    out = {}
    if "bin" in formats:
        out["bin"] = f"{prefix}.bin"
        write_neutral_fractions_binary(out["bin"], grid, x)
    if "dat" in formats:
        if nH_blocked is None:
            raise ValueError("the .dat format needs n_H (nH_blocked)")
        out["dat"] = f"{prefix}.dat"
        write_neutral_fractions_dat(out["dat"], grid, x, nH_blocked)
    unknown = set(formats) - {"dat", "bin"}
    if unknown:
        raise ValueError(f"unknown formats {sorted(unknown)} (hdf5 needs libhdf5)")
    return out


def radial_profile(records, centre=(0.0, 0.0, 0.0), bins=100, r_max=None):
    """Mean x_H in radial shells around ``centre`` from .dat records: the
    quantity scripts/plot_neutral_fraction_profile.py plots against the
    semi-analytic Stromgren profile (that script reads the file as 10 FP64
    per cell, which does not match the 60-byte records the reference
    writes; this reads the records as written)."""
    pos = records["pos"] - np.asarray(centre, dtype=np.float64)
    r = np.sqrt((pos ** 2).sum(axis=1))
    r_max = float(r.max()) if r_max is None else float(r_max)
    edges = np.linspace(0.0, r_max, bins + 1)
    idx = np.clip(np.digitize(r, edges) - 1, 0, bins - 1)
    cnt = np.bincount(idx, minlength=bins)
    tot = np.bincount(idx, weights=records["xH"], minlength=bins)
    mid = 0.5 * (edges[1:] + edges[:-1])
    with np.errstate(invalid="ignore", divide="ignore"):
        return mid, np.where(cnt > 0, tot / np.maximum(cnt, 1), np.nan)
