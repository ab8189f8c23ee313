"""The U-Net oracle (oracle/unet_oracle.py) pinned by finite differences,
and its building blocks against direct definitions.  CPU only."""
import numpy as np
import pytest

from oracle import unet_oracle as U


def test_bf16_round():
    a = np.array([1.0, 1.00390625, 1.0078125, 1.01171875, -3.14159, 0.0, 1e-40, np.inf])
    r = U.bf16_round(a)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 -> even (1); 1 + 3*2^-8 -> 1 + 2^-6
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[3] == 1.015625
    assert abs(r[4] + 3.140625) < 1e-12 and r[5] == 0.0 and r[7] == np.inf


def test_conv3_against_direct_sum():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(1, 4, 5, 6, 3))
    W = rng.normal(size=(2, 27, 3))
    b = rng.normal(size=2)
    y = U.conv3(x, W, b)
    # one output voxel by the definition
    z0, y0, x0 = 0, 2, 5
    ref = b.copy()
    for t, (dz, dy, dx) in enumerate(U.TAPS):
        z, yy, xx = z0 + dz, y0 + dy, x0 + dx
        if 0 <= z < 4 and 0 <= yy < 5 and 0 <= xx < 6:
            ref += W[:, t, :] @ x[0, z, yy, xx]
    np.testing.assert_allclose(y[0, z0, y0, x0], ref, rtol=1e-12)
    # adjoint identities: <conv(x), d> = <x, conv_input_grad(d)> = <W, weight_grad(x, d)>
    d = rng.normal(size=y.shape)
    lhs = np.sum(U.conv3(x, W) * d)
    assert abs(lhs - np.sum(x * U.conv3_input_grad(d, W))) < 1e-9 * abs(lhs)
    assert abs(lhs - np.sum(W * U.conv3_weight_grad(x, d))) < 1e-9 * abs(lhs)


def test_pool_and_upsample_adjoints():
    rng = np.random.default_rng(2)
    x = rng.normal(size=(2, 4, 4, 6, 3))
    d = rng.normal(size=(2, 2, 2, 3, 3))
    assert abs(np.sum(U.pool2(x) * d) - np.sum(x * U.pool2_grad(d))) < 1e-12
    e = rng.normal(size=(2, 4, 4, 6, 3))
    assert abs(np.sum(U.up2(d) * e) - np.sum(d * U.up2_grad(e))) < 1e-12


def test_parameter_count():
    assert U.num_params() == 199_513  # the default 12/24/48 network (~2e5)
    p = U.init_params()
    assert p.size == U.num_params()
    convs, (hw, hb) = U.split_params(p)
    assert convs[6][0].shape == (24, 27, 72) and hw.shape == (12,)


@pytest.mark.parametrize("seed,over_weight", [(0, 1.0), (1, 1.0), (2, 4.0)])
def test_oracle_gradient_matches_finite_differences(seed, over_weight):
    c = (3, 4, 5)
    rng = np.random.default_rng(seed)
    p = U.init_params(*c, seed=seed)
    p[:] += rng.normal(0, 0.05, p.size)  # non-zero biases
    feats = rng.normal(size=(2, 8, 8, 8, 3))
    target = rng.normal(size=(2, 8, 8, 8))
    net = U.UNetOracle(p, *c)
    loss, g = net.gradients(feats, target, over_weight)
    assert np.isclose(loss, net.loss(feats, target, over_weight))
    idx = rng.choice(p.size, 60, replace=False)
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (U.UNetOracle(pp, *c).loss(feats, target, over_weight) -
              U.UNetOracle(pm, *c).loss(feats, target, over_weight)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(fd), 1e-3), (i, fd, g[i])
