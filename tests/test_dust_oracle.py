"""The dust path's CPU oracle (oracle/cmi_oracle.c: cmio_propagate,
cmio_compute_optical_depth, cmio_dust_run) against the reference: the walks
bit for bit against DensitySubGrid::propagate / compute_optical_depth
(tests/golden/dust_walks.npz), the whole photon loop statistically against
the image of the reference's dust driver (tests/golden/dust_image.npz; both
made by tests/golden/make_golden.py).  CPU only."""
import math

import numpy as np
import pytest

from conftest import golden

import oracle as O
from parallelcmacionize_b200.problems import dust_sphere


@pytest.mark.parametrize("case", ["interior16", "entries8", "noncubic"])
@pytest.mark.parametrize("depth", [False, True])
def test_walks_match_reference_bit_for_bit(case, depth):
    g = golden(f"walk_{case}.npz")
    d = golden("dust_walks.npz")
    sg = O.subgrid(g["box"], g["ncell"])
    ph, dirs = g["photons"], g["in_dirs"]
    if depth:
        out_ref, res_ref = d[f"{case}_depth_out"], d[f"{case}_depth_res"]
    else:
        keep = d[f"{case}_keep"]
        ph, dirs = ph[keep], dirs[keep]
        out_ref, res_ref = d[f"{case}_prop_out"], d[f"{case}_prop_res"]
    walk = O.compute_optical_depth if depth else O.propagate
    for i in range(ph.size):
        p = ph[i: i + 1].copy()
        res, _ = walk(sg, g["nH"], g["xH"], p, int(dirs[i]))
        assert res == res_ref[i], (i, res, res_ref[i])
        assert p.tobytes() == out_ref[i: i + 1].tobytes(), i


def test_dust_exp():
    xs = -np.concatenate([np.linspace(0.0, 60.0, 3001), np.logspace(-14, 2.84, 400)])
    for x in xs:
        e = math.exp(x)
        # a few ulp of the correctly rounded value
        assert abs(O.dust_exp(x) - e) <= 4 * math.ulp(e), x
    assert O.dust_exp(-701.0) == 0.0 and O.dust_exp(0.0) == 1.0


def _rings(image, edges=np.linspace(0.0, 1.2, 7)):
    n = image.shape[0]
    ix, iy = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    r = np.hypot((ix + 0.5) / n * 2 - 1, (iy + 0.5) / n * 2 - 1)
    return np.array([image[(r >= a) & (r < b)].sum() for a, b in zip(edges[:-1], edges[1:])])


def test_photon_loop_matches_reference_image():
    """Unit-density sphere, albedo 0.5, 1e6 packets on each side: the total
    peel-off flux within 1% and the flux in 5 radial rings within 3% (the
    Monte Carlo noise of either side is 0.2-0.6% per ring at 1e6 packets)."""
    ref = golden("dust_image.npz")
    grid, nH, xH = dust_sphere(int(ref["ncell"]), int(ref["num_subgrid"]))
    lat = O.LatticeGrid(grid.box, grid.ncell, grid.num_subgrid)
    img, st = lat.dust_run(nH, xH, int(ref["num_photon"]), 11, float(ref["albedo"]),
                           [0.0, 0.0, 0.0], source_subgrid=42)
    assert st["emitted"] == st["absorbed"] + st["escaped"]  # every line ends once
    assert st["peeloffs_off_image"] == 0 and st["error_flags"] == 0
    assert abs(img.sum() / ref["image"].sum() - 1) < 0.01
    r_ours, r_ref = _rings(img), _rings(ref["image"])
    np.testing.assert_allclose(r_ours[:5], r_ref[:5], rtol=0.03)


def test_albedo_zero_gives_no_image():
    grid, nH, xH = dust_sphere(16, 2)
    lat = O.LatticeGrid(grid.box, grid.ncell, grid.num_subgrid)
    img, st = lat.dust_run(nH, xH, 5000, 3, 0.0, [0.0, 0.0, 0.0], source_subgrid=7)
    assert not img.any()
    # the forced first scattering puts every relaunched packet inside the box
    assert st["scatterings"] == 0 and st["absorbed"] == 5000 and st["escaped"] == 0
