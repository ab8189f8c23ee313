"""Result files in the reference's formats (parallelcmacionize_b200/outputs.py)
against the files the reference's own driver writes (tests/golden/outputs.npz,
made by tests/golden/make_golden.py from oracle/_ref/testDensitySubGrid_omp_files,
one thread).  CPU only."""
import os

import numpy as np

from conftest import golden
from parallelcmacionize_b200 import GridSpec
from parallelcmacionize_b200.outputs import (DAT_RECORD, cell_centres_blocked,
                                              neutral_fractions_dat, radial_profile,
                                              read_neutral_fractions_binary,
                                              read_neutral_fractions_dat,
                                              write_neutral_fractions_binary,
                                              write_neutral_fractions_dat)
from parallelcmacionize_b200.problems import PARSEC


def _grid(g):
    anchor = g["anchor_pc"] * PARSEC
    sides = g["sides_pc"] * PARSEC
    return GridSpec(box=tuple(anchor) + tuple(sides), ncell=tuple(int(v) for v in g["ncell"]),
                    num_subgrid=tuple(int(v) for v in g["num_subgrid"]))


def test_dat_record_layout():
    assert DAT_RECORD.itemsize == 60  # 5 FP64 + 5 x 4 bytes (DensitySubGrid.hpp:1793-1796)


def test_reference_dat_decodes():
    g = golden("outputs.npz")
    rec = g["dat"].view(DAT_RECORD)
    grid = _grid(g)
    assert rec.size == int(np.prod(grid.ncell))
    # x_H in the .dat equals the .bin, in the same (blocked) order
    assert np.array_equal(rec["xH"], g["bin"])
    assert np.all(rec["nH"] == 1e8)          # uniform density of the run
    assert np.all(rec["hydro"] == 0)         # NO_HYDRO: zero slots
    # cell centres: the reference's arithmetic, bit for bit
    assert np.array_equal(rec["pos"], cell_centres_blocked(grid))


def test_writers_reproduce_the_reference_files(tmp_path):
    g = golden("outputs.npz")
    grid = _grid(g)
    x = g["bin"]
    nh = np.full(x.size, 1e8)
    p = os.path.join(tmp_path, "nf.dat")
    assert write_neutral_fractions_dat(p, grid, x, nh) == g["dat"].size
    assert np.array_equal(np.fromfile(p, dtype=np.uint8), g["dat"])
    q = os.path.join(tmp_path, "nf.bin")
    write_neutral_fractions_binary(q, grid, x)
    assert np.array_equal(np.fromfile(q, dtype=np.uint8), g["bin"].view(np.uint8))
    assert np.array_equal(read_neutral_fractions_binary(q), x)
    rec = read_neutral_fractions_dat(p)
    assert np.array_equal(rec["xH"], x)


def test_dat_size_checks(tmp_path):
    g = golden("outputs.npz")
    grid = _grid(g)
    import pytest
    with pytest.raises(ValueError):
        neutral_fractions_dat(grid, np.zeros(5), np.zeros(5))
    p = os.path.join(tmp_path, "short.dat")
    np.zeros(61, dtype=np.uint8).tofile(p)
    with pytest.raises(ValueError):
        read_neutral_fractions_dat(p)


def test_radial_profile_of_a_step():
    grid = GridSpec(box=(-1.0, -1.0, -1.0, 2.0, 2.0, 2.0), ncell=(16, 16, 16),
                    num_subgrid=(2, 2, 2))
    pos = cell_centres_blocked(grid)
    r = np.sqrt((pos ** 2).sum(axis=1))
    x = np.where(r < 0.5, 1e-4, 1.0)
    rec = neutral_fractions_dat(grid, x, np.full(x.size, 1e8))
    mid, prof = radial_profile(rec, bins=8, r_max=1.0)
    np.testing.assert_allclose(prof[mid < 0.4], 1e-4, rtol=1e-12)
    np.testing.assert_allclose(prof[mid > 0.6], 1.0, rtol=1e-12)
