"""CPU oracle of the warm-start U-Net (test infrastructure only).

A plain numpy restatement, in FP64, of the network the CUDA library trains
(parallelcmacionize_b200/csrc/cmi_unet.cu): 3x3x3 convolutions with zero
padding and leaky ReLU, 2x2x2 average pooling, nearest-neighbour upsampling,
skip connections concatenated after the upsampled channels, a 1x1 output head
and the mean-squared-error loss, with the analytic backward pass.  The
network has no counterpart in the reference (it starts from x_H = 1e-6,
DensitySubGrid.hpp:544-551), so this oracle is pinned by finite differences of
its own loss (tests/test_unet_oracle.py), not by reference outputs.

``bf16=True`` rounds weights and every stored activation / gradient to BF16
(round to nearest even) at the points where the GPU stores BF16, so GPU and
oracle differ only by FP32-vs-FP64 accumulation.

Tensors are channels-last [batch, Z, Y, X, C]; parameters use the library's
order: per convolution W[co][tap][ci] (tap = (dz * 3 + dy) * 3 + dx) then
b[co]; last the head w[c1], b.
"""
from __future__ import annotations

import numpy as np

SLOPE = 0.1
NUM_FEATURES = 3  # input channels


def bf16_round(a):
    """Round to the nearest BF16 value (ties to even), returned as FP64."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    out = np.where(np.isnan(a), a, out)
    return out.astype(np.float64)


def layer_specs(c1=12, c2=24, c3=48):
    """(cout, [input segment channels]) of the ten convolutions."""
    return [(c1, [NUM_FEATURES]), (c1, [c1]), (c2, [c1]), (c2, [c2]), (c3, [c2]), (c3, [c3]),
            (c2, [c3, c2]), (c2, [c2]), (c1, [c2, c1]), (c1, [c1])]


def num_params(c1=12, c2=24, c3=48):
    n = 0
    for cout, segs in layer_specs(c1, c2, c3):
        n += cout * 27 * sum(segs) + cout
    return n + c1 + 1


def split_params(p, c1=12, c2=24, c3=48):
    """Views (W [co, 27, ci], b [co]) per convolution and the head (w, b)."""
    out, off = [], 0
    for cout, segs in layer_specs(c1, c2, c3):
        cin = sum(segs)
        W = p[off: off + cout * 27 * cin].reshape(cout, 27, cin)
        off += cout * 27 * cin
        b = p[off: off + cout]
        off += cout
        out.append((W, b))
    hw = p[off: off + c1]
    hb = p[off + c1: off + c1 + 1]
    return out, (hw, hb)


def init_params(c1=12, c2=24, c3=48, seed=0):
    """He-normal weights, zero biases (the initialisation the host uses)."""
    rng = np.random.default_rng(seed)
    parts = []
    for cout, segs in layer_specs(c1, c2, c3):
        cin = sum(segs)
        parts.append(rng.normal(0.0, np.sqrt(2.0 / (27 * cin)), cout * 27 * cin))
        parts.append(np.zeros(cout))
    parts.append(rng.normal(0.0, np.sqrt(1.0 / c1), c1))
    parts.append(np.zeros(1))
    return np.concatenate(parts)


def _shift(x, dz, dy, dx):
    """x[., z+dz, y+dy, x+dx, .] with zeros outside."""
    B, Z, Y, X, C = x.shape
    out = np.zeros_like(x)
    zs, ys, xs = slice(max(0, -dz), min(Z, Z - dz)), slice(max(0, -dy), min(Y, Y - dy)), \
        slice(max(0, -dx), min(X, X - dx))
    zt, yt, xt = slice(max(0, dz), min(Z, Z + dz)), slice(max(0, dy), min(Y, Y + dy)), \
        slice(max(0, dx), min(X, X + dx))
    out[:, zs, ys, xs, :] = x[:, zt, yt, xt, :]
    return out


TAPS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def conv3(x, W, b=None):
    """y[v, co] = sum_{tap, ci} W[co, tap, ci] x[v + tap, ci] (+ b)."""
    y = np.zeros(x.shape[:4] + (W.shape[0],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += _shift(x, dz, dy, dx) @ W[:, t, :].T
    if b is not None:
        y += b
    return y


def conv3_input_grad(dy, W):
    """dx[v, ci] = sum_{tap, co} W[co, tap, ci] dy[v - tap, co]."""
    dx = np.zeros(dy.shape[:4] + (W.shape[2],))
    for t, (dz, dyy, dxx) in enumerate(TAPS):
        dx += _shift(dy @ W[:, t, :], -dz, -dyy, -dxx)
    return dx


def conv3_weight_grad(x, dy):
    """dW[co, tap, ci] = sum_v dy[v, co] x[v + tap, ci]."""
    co, ci = dy.shape[-1], x.shape[-1]
    dW = np.zeros((co, 27, ci))
    d2 = dy.reshape(-1, co)
    for t, (dz, dyy, dxx) in enumerate(TAPS):
        dW[:, t, :] = d2.T @ _shift(x, dz, dyy, dxx).reshape(-1, ci)
    return dW


def leaky(a):
    return np.where(a > 0, a, SLOPE * a)


def pool2(x):
    B, Z, Y, X, C = x.shape
    return x.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(2, 4, 6))


def pool2_grad(d):
    return np.repeat(np.repeat(np.repeat(d, 2, axis=1), 2, axis=2), 2, axis=3) / 8.0


def up2(x):
    return np.repeat(np.repeat(np.repeat(x, 2, axis=1), 2, axis=2), 2, axis=3)


def up2_grad(d):
    B, Z, Y, X, C = d.shape
    return d.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(2, 4, 6))


class UNetOracle:
    def __init__(self, params, c1=12, c2=24, c3=48, bf16=False):
        self.c = (c1, c2, c3)
        self.bf16 = bf16
        self.params = np.asarray(params, dtype=np.float64)
        convs, (hw, hb) = split_params(self.params, c1, c2, c3)
        r = bf16_round if bf16 else (lambda a: a)
        self.W = [r(W) for W, _ in convs]      # the GPU packs weights as BF16
        self.b = [b.copy() for _, b in convs]  # biases stay FP32
        self.hw, self.hb = hw.copy(), hb.copy()

    def _q(self, a):
        return bf16_round(a) if self.bf16 else a

    def forward(self, feats):
        """feats [B, Z, Y, X, 3] -> prediction [B, Z, Y, X]; keeps activations."""
        q = self._q
        W, b = self.W, self.b
        s = {}
        s["x0"] = q(feats)
        s["e1a"] = q(leaky(conv3(s["x0"], W[0], b[0])))
        s["e1b"] = q(leaky(conv3(s["e1a"], W[1], b[1])))
        s["p1"] = q(pool2(s["e1b"]))
        s["e2a"] = q(leaky(conv3(s["p1"], W[2], b[2])))
        s["e2b"] = q(leaky(conv3(s["e2a"], W[3], b[3])))
        s["p2"] = q(pool2(s["e2b"]))
        s["ba"] = q(leaky(conv3(s["p2"], W[4], b[4])))
        s["bb"] = q(leaky(conv3(s["ba"], W[5], b[5])))
        s["cat2"] = np.concatenate([up2(s["bb"]), s["e2b"]], axis=-1)
        s["d2a"] = q(leaky(conv3(s["cat2"], W[6], b[6])))
        s["d2b"] = q(leaky(conv3(s["d2a"], W[7], b[7])))
        s["cat1"] = np.concatenate([up2(s["d2b"]), s["e1b"]], axis=-1)
        s["d1a"] = q(leaky(conv3(s["cat1"], W[8], b[8])))
        s["d1b"] = q(leaky(conv3(s["d1a"], W[9], b[9])))
        s["pred"] = s["d1b"] @ self.hw + self.hb[0]
        self.s = s
        return s["pred"]

    @staticmethod
    def _weights(diff, over_weight):
        """Per-voxel loss weights: over_weight where the prediction is above
        the target (the library's cmi_unet_set_loss_weight), else 1."""
        return np.where(diff > 0, over_weight, 1.0)

    def loss(self, feats, target, over_weight=1.0):
        d = self.forward(feats) - target
        return float(np.mean(self._weights(d, over_weight) * d ** 2))

    def gradients(self, feats, target, over_weight=1.0):
        """(loss, gradient in the library's parameter order)."""
        q = self._q
        pred = self.forward(feats)
        s = self.s
        n = pred.size
        c1, c2, c3 = self.c
        w = self._weights(pred - target, over_weight)
        gp = 2.0 * w * (pred - target) / n
        g_hw = np.einsum("bzyxc,bzyx->c", s["d1b"], gp)
        g_hb = np.array([gp.sum()])
        gW = [None] * 10
        gb = [None] * 10

        def back(i, x, y, dy):
            dy = q(np.where(y > 0, dy, SLOPE * dy))
            gW[i] = conv3_weight_grad(x, dy)
            gb[i] = dy.sum(axis=(0, 1, 2, 3))
            return dy

        d = q(gp[..., None] * self.hw)
        dy = back(9, s["d1a"], s["d1b"], d)
        d = q(conv3_input_grad(dy, self.W[9]))
        dy = back(8, s["cat1"], s["d1a"], d)
        dcat1 = q(conv3_input_grad(dy, self.W[8]))
        d = q(up2_grad(dcat1[..., :c2]))
        dy = back(7, s["d2a"], s["d2b"], d)
        d = q(conv3_input_grad(dy, self.W[7]))
        dy = back(6, s["cat2"], s["d2a"], d)
        dcat2 = q(conv3_input_grad(dy, self.W[6]))
        d = q(up2_grad(dcat2[..., :c3]))
        dy = back(5, s["ba"], s["bb"], d)
        d = q(conv3_input_grad(dy, self.W[5]))
        dy = back(4, s["p2"], s["ba"], d)
        dp2 = q(conv3_input_grad(dy, self.W[4]))
        d = q(dcat2[..., c3:] + pool2_grad(dp2))
        dy = back(3, s["e2a"], s["e2b"], d)
        d = q(conv3_input_grad(dy, self.W[3]))
        dy = back(2, s["p1"], s["e2a"], d)
        dp1 = q(conv3_input_grad(dy, self.W[2]))
        d = q(dcat1[..., c2:] + pool2_grad(dp1))
        dy = back(1, s["e1a"], s["e1b"], d)
        d = q(conv3_input_grad(dy, self.W[1]))
        back(0, s["x0"], s["e1a"], d)
        parts = []
        for i in range(10):
            parts.append(gW[i].ravel())
            parts.append(gb[i])
        parts.append(g_hw)
        parts.append(g_hb)
        loss = float(np.mean(w * (pred - target) ** 2))
        return loss, np.concatenate(parts)
