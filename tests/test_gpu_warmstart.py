"""What the trained warm-start network gains over the plain method
(parallelcmacionize_b200/warmstart.py, shipped weights
parallelcmacionize_b200/weights/warmstart_unet64.npz, trained on seeds
100000-101599 of the log-normal 64^3 generator).

On held-out seeds: iterations to the plain method's convergence criterion
(mean |delta x_H| < 0.01), wall time, and the accuracy of the converged field
against a long plain run (24 iterations, x_H averaged over the last 6)."""
import numpy as np
import pytest

from parallelcmacionize_b200.warmstart import (DEFAULT_WEIGHTS, UNet, generate_runs,
                                               run_configs, time_to_converge)

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net():
    n = UNet.load(DEFAULT_WEIGHTS)
    yield n
    n.close()


def test_shipped_weights_describe_the_network(net):
    assert net.num_params == 199_513
    assert float(net.meta["val_mse"]) < 0.1 * float(net.meta["baseline_mse"])


@pytest.mark.parametrize("seed", [101_990, 101_991])
def test_warm_start_converges_faster_to_the_same_field(net, seed):
    g, nH = run_configs([seed])[0]
    _, _, labels, _ = generate_runs([seed], batch=1)
    ref = 10.0 ** labels[0].astype(np.float64)
    r = time_to_converge(net, g, nH, x_reference=ref, tolerance=0.01)
    assert r["plain"]["converged"] and r["warm"]["converged"]
    # at least 3 iterations fewer (plain needs 6-8 on this generator)
    assert r["warm"]["iterations"] <= r["plain"]["iterations"] - 3, r
    # as accurate as the plain method's own converged field, against the long
    # run (two plain runs share their start and so their remaining convergence
    # error; the warm start reaches the fixed point from another side, so its
    # distance to a plain run is no accuracy measure)
    assert r["warm"]["error_vs_reference"] <= r["plain"]["error_vs_reference"] + 0.005, r
    # wall time, features and network included (the bench measures it precisely)
    assert r["speedup"] > 1.5, r
