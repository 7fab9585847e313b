"""Float reference of the learned warm start's MLP for checking the tensor-core kernels: numpy f32
arithmetic with the operands rounded to bf16 exactly where the GPU rounds them (inputs, weights,
hidden activations, and the backward pass's tensor-core operands)."""
import numpy as np

IN, IN_PAD, H = 24, 32, 128
W1, B1 = 0, H * IN_PAD
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H * H
W4 = B3 + H
B4 = W4 + 16 * H
N_PARAMS = B4 + 16


def bf16(x):
    """Round f32 to the nearest bf16 (ties to even), returned as f32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(np.shape(x))


def unpack(w):
    return (w[W1:B1].reshape(H, IN_PAD), w[B1:W2], w[W2:B2].reshape(H, H), w[B2:W3], w[W3:B3].reshape(H, H),
            w[B3:W4], w[W4:B4].reshape(16, H), w[B4:N_PARAMS])


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(w, feats):
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(w)
    x = np.zeros((len(feats), IN_PAD), np.float32)
    x[:, :IN] = feats
    x = bf16(x)
    z1 = x @ bf16(w1).T + b1
    h1 = bf16(silu(z1))
    z2 = h1 @ bf16(w2).T + b2
    h2 = bf16(silu(z2))
    z3 = h2 @ bf16(w3).T + b3
    h3 = bf16(silu(z3))
    y = h3 @ bf16(w4).T + b4
    return y[:, :3], (x, z1, h1, z2, h2, z3, h3, y)


def gradients(w, feats, targets):
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(w)
    y3, (x, z1, h1, z2, h2, z3, h3, y) = forward(w, feats)
    n = len(feats)
    dy = np.zeros((n, 16), np.float32)
    dy[:, :3] = 2.0 * (y3 - targets) / (3.0 * n)
    g = np.zeros(N_PARAMS, np.float32)
    dyb = bf16(dy)
    g[W4:B4] = (h3.T @ dyb).T.reshape(-1)
    g[B4:N_PARAMS] = dy.sum(0)
    dh = dyb @ bf16(w4)
    gz = bf16(dh * dsilu(z3))
    g[W3:B3] = (gz.T @ h2).reshape(-1)
    g[B3:W4] = gz.sum(0)
    dh = gz @ bf16(w3)
    gz = bf16(dh * dsilu(z2))
    g[W2:B2] = (gz.T @ h1).reshape(-1)
    g[B2:W3] = gz.sum(0)
    dh = gz @ bf16(w2)
    gz = bf16(dh * dsilu(z1))
    g[W1:B1] = (gz.T @ x).reshape(-1)
    g[B1:W2] = gz.sum(0)
    loss = float(((y3 - targets) ** 2).mean())
    return g, loss
