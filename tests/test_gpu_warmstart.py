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


def test_finer_grids_are_predicted_at_the_training_resolution(net):
    """A 128^3 grid: n_H is block-averaged to 64^3 (checked against numpy),
    the network predicts there and the prediction is upsampled (nearest)."""
    import ctypes as C

    from parallelcmacionize_b200 import GridSpec, _lib
    from parallelcmacionize_b200.problems import BOX_10PC, lognormal_density, random_sources
    from parallelcmacionize_b200.warmstart import predict_log_xH

    fine = lognormal_density(128, seed=3)
    srcs = random_sources(BOX_10PC, 3, seed=4)
    g128 = GridSpec(box=BOX_10PC, ncell=(128,) * 3, num_subgrid=(8,) * 3, sources=srcs)
    g64 = GridSpec(box=BOX_10PC, ncell=(64,) * 3, num_subgrid=(4,) * 3, sources=srcs)
    dev = torch.from_numpy(fine.ravel().copy()).cuda()
    coarse = torch.empty(64 ** 3, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check_unet(net._L.cmi_unet_block_mean(net._h, C.c_void_p(dev.data_ptr()),
                                               (C.c_int32 * 3)(128, 128, 128), 2,
                                               C.c_void_p(coarse.data_ptr())))
    ref = fine.reshape(64, 2, 64, 2, 64, 2).mean(axis=(1, 3, 5))
    np.testing.assert_allclose(coarse.cpu().numpy().reshape(64, 64, 64), ref, rtol=1e-14)
    p128 = predict_log_xH(net, g128, dev).cpu().numpy().reshape(128, 128, 128)
    p64 = predict_log_xH(net, g64, coarse).cpu().numpy().reshape(64, 64, 64)
    up = np.repeat(np.repeat(np.repeat(p64, 2, 0), 2, 1), 2, 2)
    assert np.array_equal(p128, up)


def test_large_grid_warm_start_converges_faster_to_the_same_field():
    """The 256^3 generator (sigma_ln = 1.5, 16 sources, 1e8 packets), a seed the
    256^3 network did not train on: at least 3 plain iterations fewer, and the
    converged field as close to the long run as the plain method's (within
    0.004; both are about 0.015 from it)."""
    from parallelcmacionize_b200.problems import large_config
    from parallelcmacionize_b200.warmstart import reference_field, weights_for

    g, nH = large_config(seed=7)
    assert weights_for(g).endswith("warmstart_unet256.npz")
    with UNet.load(weights_for(g)) as n256:
        assert n256.ratio_factor == 4 and float(n256.meta["over_weight"]) > 1
        ref = reference_field(g, nH)
        r = time_to_converge(n256, g, nH, x_reference=ref, tolerance=0.01)
    assert r["plain"]["converged"] and r["warm"]["converged"], r
    assert r["warm"]["iterations"] <= r["plain"]["iterations"] - 3, r
    assert r["warm"]["error_vs_reference"] <= r["plain"]["error_vs_reference"] + 0.004, r
    assert r["speedup"] > 1.5, r
