"""FP32 CPU oracle of the prefilter MLP -- TEST INFRASTRUCTURE ONLY.

The prefilter has no reference counterpart; this restates its forward pass
and its binary-cross-entropy gradients with numpy in FP32, rounding to BF16
(round to nearest even) at exactly the points where the GPU kernels hold
BF16 values: the weight copies W1, W2 (GEMM operands), the layer-1 and
layer-2 activations, and the back-propagated dZ2 and dZ1 (GEMM operands).
Only the order of FP32 accumulation differs from the tensor cores.

Parameter vector (99073 floats): W1[256][128] (inputs past 4k are zero),
b1[256], W2[256][256] ([out][in]), b2[256], w3[256], b3.
"""
import numpy as np

OFF = {"W1": 0, "b1": 32768, "W2": 33024, "b2": 98560, "w3": 98816, "b3": 99072, "count": 99073}


def bf16(x):
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(theta):
    t = np.asarray(theta, dtype=np.float32)
    return (t[0:32768].reshape(256, 128), t[32768:33024], t[33024:98560].reshape(256, 256), t[98560:98816],
            t[98816:99072], float(t[99072]))


def onehot(kmers, k):
    km = np.asarray(kmers, dtype=np.uint64)
    X = np.zeros((km.size, 128), dtype=np.float32)
    for i in range(k):
        c = ((km >> np.uint64(62 - 2 * i)) & np.uint64(3)).astype(np.int64)
        X[np.arange(km.size), 4 * i + c] = 1.0
    return X


def forward(theta, kmers, k):
    W1, b1, W2, b2, w3, b3 = unpack(theta)
    X = onehot(kmers, k)
    Z1 = X @ bf16(W1).T
    H1 = bf16(np.maximum(Z1 + b1, 0))
    Z2 = H1 @ bf16(W2).T
    H2 = bf16(np.maximum(Z2 + b2, 0))
    z = H2 @ w3 + b3
    return z, (X, H1, H2)


def loss_and_grad(theta, kmers, labels, k):
    W1, b1, W2, b2, w3, b3 = unpack(theta)
    z, (X, H1, H2) = forward(theta, kmers, k)
    y = np.asarray(labels, dtype=np.float32)
    B = y.size
    loss = float(np.mean(np.logaddexp(0, z) - y * z))
    dz = (1.0 / (1.0 + np.exp(-z)) - y) / B
    dZ2 = bf16(np.where(H2 > 0, dz[:, None] * w3[None, :], 0.0))
    dH1 = dZ2 @ bf16(W2)
    dZ1 = bf16(np.where(H1 > 0, dH1, 0.0))
    g = np.zeros(OFF["count"], dtype=np.float32)
    g[0:32768] = (dZ1.T @ X).reshape(-1)
    g[32768:33024] = dZ1.sum(0)
    g[33024:98560] = (dZ2.T @ H1).reshape(-1)
    g[98560:98816] = dZ2.sum(0)
    g[98816:99072] = (dz[:, None] * H2).sum(0)
    g[99072] = dz.sum()
    return loss, g


def init_like(seed=0, k=31):
    """Parameters of the scale the trainer starts from (U(+-1/sqrt(fan_in)))."""
    rng = np.random.default_rng(seed)
    t = np.zeros(OFF["count"], dtype=np.float32)
    W1 = rng.uniform(-1, 1, (256, 128)) / np.sqrt(4 * k)
    W1[:, 4 * k:] = 0
    t[0:32768] = W1.reshape(-1)
    t[32768:33024] = rng.uniform(-1, 1, 256) / np.sqrt(4 * k)
    t[33024:98560] = rng.uniform(-1, 1, 65536) / 16
    t[98560:98816] = rng.uniform(-1, 1, 256) / 16
    t[98816:99072] = rng.uniform(-1, 1, 256) / 16
    t[99072] = 0.01
    return t
