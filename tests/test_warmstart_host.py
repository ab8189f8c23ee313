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


def test_weights_selection_and_large_weights_metadata():
    from parallelcmacionize_b200 import GridSpec
    from parallelcmacionize_b200.problems import BOX_10PC
    from parallelcmacionize_b200.warmstart import DEFAULT_WEIGHTS, LARGE_WEIGHTS, weights_for

    def grid(n):
        return GridSpec(box=BOX_10PC, ncell=(n,) * 3, num_subgrid=(n // 16,) * 3)
    assert weights_for(grid(256)) == LARGE_WEIGHTS
    assert weights_for(grid(64)) == DEFAULT_WEIGHTS
    assert weights_for(grid(128)) == DEFAULT_WEIGHTS  # predicted on the 64^3 block mean
    d = np.load(LARGE_WEIGHTS)
    assert int(d["ncell"]) == 256 and int(d["ratio_factor"]) == 4
    assert d["params"].size == 199_513 and float(d["over_weight"]) > 1
    # trained and validated on seeds away from the bench's and the tests' (7, 8)
    assert int(d["train_seeds"][0]) >= 300_000 and int(d["val_seeds"][0]) >= 300_000
    assert float(d["val_mse"]) < 0.25 * float(d["baseline_mse"])
