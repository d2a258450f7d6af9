"""FP64 numpy restatement of the diagonal MLP (test infrastructure only).

Same layout and loss as loadsg_b200/csrc/lsg_mlp.cu: W1[64][F] b1 W2[64][64] b2
W3[64][64] b3 W4[64] b4, ReLU hidden layers, loss mean_r (log softplus(o_r) -
y_r)^2.  Weights are rounded to BF16 (round to nearest even) as the CUDA
forward/backward passes use them, and so are the inputs of the three hidden
layers (the tensor cores multiply BF16 by BF16: the features X and the
activations a1, a2); biases, a3 and the output layer stay in floating point.
Used to check the CUDA forward pass and gradients."""
import numpy as np

H = 64


def layout(F):
    sizes = [("W1", H * F), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H), ("b3", H), ("W4", H), ("b4", 1)]
    off, out = 0, {}
    for k, n in sizes:
        out[k] = (off, n)
        off += n
    return out, off


def bf16_round(a):
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p, F):
    lay, _ = layout(F)
    g = {k: p[o:o + n] for k, (o, n) in lay.items()}
    return (bf16_round(g["W1"]).astype(np.float64).reshape(H, F), g["b1"].astype(np.float64),
            bf16_round(g["W2"]).astype(np.float64).reshape(H, H), g["b2"].astype(np.float64),
            bf16_round(g["W3"]).astype(np.float64).reshape(H, H), g["b3"].astype(np.float64),
            bf16_round(g["W4"]).astype(np.float64), float(g["b4"][0]))


def forward(p, X):
    F = X.shape[1]
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, F)
    X = bf16_round(X).astype(np.float64)
    a1 = bf16_round(np.maximum(X @ W1.T + b1, 0)).astype(np.float64)
    a2 = bf16_round(np.maximum(a1 @ W2.T + b2, 0)).astype(np.float64)
    a3 = np.maximum(a2 @ W3.T + b3, 0)
    return a3 @ W4 + b4, (X, a1, a2, a3)


def softplus(o):
    return np.where(o > 20, o, np.log1p(np.exp(np.minimum(o, 20))))


def loss_and_grad(p, X, Y):
    """Mean loss and its gradient with respect to the (BF16-rounded) weights."""
    F = X.shape[1]
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, F)
    o, (X, a1, a2, a3) = forward(p, X)
    n = len(Y)
    sp = softplus(o)
    e = np.log(sp) - Y
    loss = float(np.mean(e * e))
    sig = 1 / (1 + np.exp(-o))
    dout = 2 * e * sig / sp / n
    gW4 = a3.T @ dout
    gb4 = dout.sum()
    d3 = np.outer(dout, W4) * (a3 > 0)
    gW3 = d3.T @ a2
    gb3 = d3.sum(0)
    d2 = (d3 @ W3) * (a2 > 0)
    gW2 = d2.T @ a1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (a1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3, gW4, [gb4]])
    return loss, g
