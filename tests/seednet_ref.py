"""CPU reference of the seed network's forward and backward passes (numpy, float64),
the checker of the library's training kernels. The parameter layout is the library's:
W1[32][64] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[64][8] b4[8], W[k][n] with k
the input and n the output unit; the loss per pair is (s - s*)^2 + (t - t*)^2 +
0.1 (d - d*)^2 over outputs 0..2, averaged over the pairs."""
import numpy as np

IN_P, H, OUT_P = 32, 64, 8
SHAPES = [("W1", (IN_P, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
          ("W4", (H, OUT_P)), ("b4", (OUT_P,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
LOSS_W = np.array([1.0, 1.0, 0.1])


def unpack(theta):
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def pack(parts):
    return np.concatenate([parts[name].ravel() for name, _ in SHAPES])


def forward(theta, x):
    p = unpack(theta)
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ p["W1"] + p["b1"], 0)
    h2 = np.maximum(h1 @ p["W2"] + p["b2"], 0)
    h3 = np.maximum(h2 @ p["W3"] + p["b3"], 0)
    out = h3 @ p["W4"] + p["b4"]
    return out, (x, h1, h2, h3)


def loss_and_grad(theta, x, y):
    p = unpack(theta)
    out, (x0, h1, h2, h3) = forward(theta, x)
    n = len(x0)
    diff = out[:, :3] - np.asarray(y, dtype=np.float64)[:, :3]
    loss = float((LOSS_W * diff * diff).sum() / n)
    d_out = np.zeros_like(out)
    d_out[:, :3] = 2.0 * LOSS_W * diff / n
    g = {"W4": h3.T @ d_out, "b4": d_out.sum(0)}
    d3 = (d_out @ p["W4"].T) * (h3 > 0)
    g["W3"], g["b3"] = h2.T @ d3, d3.sum(0)
    d2 = (d3 @ p["W3"].T) * (h2 > 0)
    g["W2"], g["b2"] = h1.T @ d2, d2.sum(0)
    d1 = (d2 @ p["W2"].T) * (h1 > 0)
    g["W1"], g["b1"] = x0.T @ d1, d1.sum(0)
    return loss, pack(g)


def loss_only(theta, x, y):
    out, _ = forward(theta, x)
    diff = out[:, :3] - np.asarray(y, dtype=np.float64)[:, :3]
    return float((LOSS_W * diff * diff).sum() / len(diff))
