"""CPU restatement of the learned router (test checker only): the 6 -> 32 ->
32 -> 1 GELU network packed as W1[32][6], b1[32], W2[32][32], b2[32], w3[32],
b3; its forward pass in FP64, a BF16-operand forward pass matching the
tensor-core path (operands rounded to BF16, FP32 accumulation), the analytic
gradient of the weighted binary cross-entropy, and a central finite-difference
gradient for checking the analytic one."""
import numpy as np

H, NF = 32, 6
NW = H * NF + H + H * H + H + H + 1


def unpack(w):
    w = np.asarray(w, np.float64)
    o = 0
    W1 = w[o:o + H * NF].reshape(H, NF); o += H * NF
    b1 = w[o:o + H]; o += H
    W2 = w[o:o + H * H].reshape(H, H); o += H * H
    b2 = w[o:o + H]; o += H
    w3 = w[o:o + H]; o += H
    b3 = w[o]
    return W1, b1, W2, b2, w3, b3


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    u = 0.7978845608028654 * (x + 0.044715 * x ** 3)
    th = np.tanh(u)
    du = 0.7978845608028654 * (1.0 + 3 * 0.044715 * x * x)
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * du


def init_weights(seed=0):
    rng = np.random.default_rng(seed)
    W1 = rng.normal(0, np.sqrt(2.0 / NF), (H, NF))
    W2 = rng.normal(0, np.sqrt(2.0 / H), (H, H))
    w3 = rng.normal(0, np.sqrt(1.0 / H), H)
    return np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, [0.0]]).astype(np.float32)


def forward(w, x):
    W1, b1, W2, b2, w3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    h1 = gelu(x @ W1.T + b1)
    h2 = gelu(h1 @ W2.T + b2)
    return h2 @ w3 + b3


def bf16(a):
    """Round-to-nearest-even to BF16, returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def forward_bf16(w, x):
    """Operands (features, W1, layer-1 activations, W2) rounded to BF16;
    sums in FP32; biases and the last layer in FP32."""
    W1, b1, W2, b2, w3, b3 = [np.asarray(v, np.float32) for v in unpack(w)]
    xb = bf16(x).astype(np.float32)
    z1 = xb @ bf16(W1).T + b1
    h1 = bf16(gelu(z1.astype(np.float64)).astype(np.float32))
    z2 = h1 @ bf16(W2).T + b2
    h2 = gelu(z2.astype(np.float64))
    return h2 @ w3.astype(np.float64) + float(b3)


def loss_and_grad(w, x, y, pos_weight=1.0):
    """Mean of pw*y*softplus(-z) + (1-y)*softplus(z) and its gradient."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    n = len(y)
    z1 = x @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    z = h2 @ w3 + b3
    sp_pos = np.logaddexp(0.0, -z)
    sp_neg = np.logaddexp(0.0, z)
    loss = np.mean(pos_weight * y * sp_pos + (1 - y) * sp_neg)
    sig = 1.0 / (1.0 + np.exp(-z))
    dz = (pos_weight * y * (sig - 1.0) + (1 - y) * sig) / n
    gw3 = h2.T @ dz
    gb3 = dz.sum()
    dz2 = np.outer(dz, w3) * gelu_grad(z2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, g


def fd_grad(w, x, y, idx, pos_weight=1.0, h=1e-6):
    w = np.asarray(w, np.float64)
    out = []
    for i in idx:
        wp = w.copy(); wp[i] += h
        wm = w.copy(); wm[i] -= h
        out.append((loss_and_grad(wp, x, y, pos_weight)[0] - loss_and_grad(wm, x, y, pos_weight)[0]) / (2 * h))
    return np.array(out)
