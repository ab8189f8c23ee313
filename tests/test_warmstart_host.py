"""Host-side pieces of the warm start (parallelcmacionize_b200/warmstart.py)
that need no GPU."""
import numpy as np

from parallelcmacionize_b200 import GridSpec
from parallelcmacionize_b200.warmstart import flux_proxy, iterations_to_tolerance, run_configs


def test_iterations_to_tolerance():
    dx = np.array([[0.5, 0.3, 0.2], [0.2, 0.009, 0.3], [0.008, 0.005, 0.3], [0.02, 0.004, 0.3]])
    assert iterations_to_tolerance(dx, 0.01).tolist() == [3, 2, 0]
    # min_iterations: the first iteration never counts
    dx0 = np.array([[0.001], [0.5], [0.002]])
    assert iterations_to_tolerance(dx0, 0.01).tolist() == [3]
    assert iterations_to_tolerance(dx0, 0.01, min_iterations=1).tolist() == [1]


def test_flux_proxy_point_source():
    L = 1e49
    g = GridSpec(box=(-1.0, -1.0, -1.0, 2.0, 2.0, 2.0), ncell=(4, 4, 4), num_subgrid=(1, 1, 1),
                 sources=[(0.0, 0.0, 0.0, L)])
    f = flux_proxy(g)
    # cell centres at +-0.25, +-0.75: the inner 8 cells are at r = sqrt(3) * 0.25
    r = np.sqrt(3) * 0.25
    assert np.isclose(f[1, 1, 1], np.log10(L / (4 * np.pi * r * r)))
    assert np.allclose(f, f[::-1, ::-1, ::-1])  # symmetric about the source
    # r clamped to half a cell
    g2 = GridSpec(box=g.box, ncell=g.ncell, num_subgrid=g.num_subgrid,
                  sources=[(0.25, 0.25, 0.25, L)])
    assert np.isclose(flux_proxy(g2)[2, 2, 2] - np.log10(L), -np.log10(4 * np.pi * 0.25 ** 2),
                      atol=0.05)


def test_run_configs_shapes():
    cfgs = run_configs([5, 6], ncell=32, packets_per_cell=2.5)
    assert len(cfgs) == 2
    g, nH = cfgs[0]
    assert g.ncell == (32, 32, 32) and g.num_subgrid == (2, 2, 2)
    assert g.num_photon == int(2.5 * 32 ** 3) and len(g.sources) == 4
    assert nH.shape == (32 ** 3,) and np.all(nH > 0)
    # seeds differ
    assert not np.array_equal(nH, cfgs[1][1])
