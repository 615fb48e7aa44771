"""NumPy reference of the schedule MLP (16 -> 64 -> 64 -> 2, ReLU, MSE):
forward pass and analytic gradient, the CPU checker of the CUDA kernels.
Parameter layout: W1[16][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2],
mean[16], std[16]."""
import numpy as np

I, H, O = 16, 64, 2


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((I, H), (H,), (H, H), (H,), (H, O), (O,), (I,), (I,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def forward(p, x_std):
    W1, b1, W2, b2, W3, b3, _, _ = unpack(p)
    a1 = x_std @ W1 + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0)
    return h2 @ W3 + b3, (h1, h2)


def standardise(p, x):
    *_, mean, std = unpack(p)
    return (np.asarray(x, np.float64) - mean) / std


def loss_and_grad(p, x_std, t):
    """Mean over samples of the squared error summed over outputs, and its
    gradient w.r.t. W1..b3 flattened in blob order."""
    W1, b1, W2, b2, W3, b3, _, _ = unpack(p)
    x_std = np.asarray(x_std, np.float64)
    t = np.asarray(t, np.float64)
    B = x_std.shape[0]
    y, (h1, h2) = forward(p, x_std)
    e = y - t
    loss = (e ** 2).sum() / B
    dy = 2 * e / B
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    d2 = (dy @ W3.T) * (h2 > 0)
    gW2 = h1.T @ d2
    gb2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    gW1 = x_std.T @ d1
    gb1 = d1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
