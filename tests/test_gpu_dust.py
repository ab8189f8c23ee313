"""The dust path on the GPU (cmi_dust_run) against the oracle's restatement
with the same counter-based draws (oracle cmio_dust_run: every count exact,
the image within FP64 summation-order rounding) and against the image of the
reference's own dust driver (tests/golden/dust_image.npz, statistically)."""
import numpy as np
import pytest

from conftest import golden

import oracle as O
from parallelcmacionize_b200 import CMIError, GridSpec, TransportEngine
from parallelcmacionize_b200.problems import dust_sphere

pytestmark = pytest.mark.gpu


def _gpu(grid, nH, xH, *args, **kw):
    with TransportEngine(grid) as eng:
        eng.set_fields(0, nH, xH)
        return eng.dust_image(0, *args, **kw)


def _source_subgrid(grid, src):
    b, ns = np.asarray(grid.box), grid.num_subgrid
    si = [min(int((src[a] - b[a]) / b[3 + a] * ns[a]), ns[a] - 1) for a in range(3)]
    return (si[0] * ns[1] + si[1]) * ns[2] + si[2]


def _compare(grid, nH, xH, n, albedo, src, npix, seed):
    img, st = _gpu(grid, nH, xH, n, albedo, source=src, npix=npix, seed=seed)
    lat = O.LatticeGrid(grid.box, grid.ncell, grid.num_subgrid)
    oimg, ost = lat.dust_run(nH, xH, n, seed, albedo, src, _source_subgrid(grid, src), npix)
    assert st == ost
    # per-pixel sums of the same terms in another order (FP64 atomics)
    np.testing.assert_allclose(img, oimg, rtol=1e-10, atol=1e-18)
    return img, st


def test_sphere_matches_oracle():
    grid, nH, xH = dust_sphere(32, 4)
    img, st = _compare(grid, nH, xH, 200_000, 0.5, (0.0, 0.0, 0.0), (101, 101), 5)
    assert st["scatterings"] > 0.6 * st["emitted"] and img.sum() > 0


def test_uneven_grid_matches_oracle():
    """Non-cubic cells and subgrids, a log-normal medium, an off-centre source,
    a rectangular image and a high albedo (many generations)."""
    rng = np.random.default_rng(4)
    grid = GridSpec(box=(-1.0, -0.5, -2.0, 2.0, 1.5, 3.0), ncell=(24, 16, 32),
                    num_subgrid=(3, 2, 4))
    nH = np.exp(rng.normal(0.0, 1.0, grid.num_cells)) * 0.8
    xH = rng.uniform(0.2, 1.0, grid.num_cells)
    _, st = _compare(grid, nH, xH, 50_000, 0.85, (0.3, 0.1, -0.7), (64, 48), 9)
    assert st["generations"] > 5


def _rings(image, edges=np.linspace(0.0, 1.2, 7)):
    n = image.shape[0]
    ix, iy = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    r = np.hypot((ix + 0.5) / n * 2 - 1, (iy + 0.5) / n * 2 - 1)
    return np.array([image[(r >= a) & (r < b)].sum() for a, b in zip(edges[:-1], edges[1:])])


def test_sphere_matches_reference_image():
    """1e6 packets on each side: total peel-off flux within 1%, the flux of
    five radial rings within 3% (Monte Carlo noise 0.2-0.6% per ring)."""
    ref = golden("dust_image.npz")
    grid, nH, xH = dust_sphere(int(ref["ncell"]), int(ref["num_subgrid"]))
    img, st = _gpu(grid, nH, xH, int(ref["num_photon"]), float(ref["albedo"]), seed=21)
    assert st["emitted"] == st["absorbed"] + st["escaped"]
    assert abs(img.sum() / ref["image"].sum() - 1) < 0.01
    np.testing.assert_allclose(_rings(img)[:5], _rings(ref["image"])[:5], rtol=0.03)


def test_invalid_arguments():
    grid, nH, xH = dust_sphere(16, 2)
    with TransportEngine(grid) as eng:
        eng.set_fields(0, nH, xH)
        for kw in ({"albedo": 1.0}, {"albedo": -0.1}, {"num_photon": 0},
                   {"source": (2.0, 0.0, 0.0)}, {"npix": (0, 10)}):
            args = {"num_photon": 100, "albedo": 0.5, **kw}
            n, a = args.pop("num_photon"), args.pop("albedo")
            with pytest.raises(CMIError):
                eng.dust_image(0, n, a, **args)
