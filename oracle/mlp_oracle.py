"""CPU oracle of the learned WENO weights network (TEST INFRASTRUCTURE ONLY).

The network maps a stencil normalised to its local range (the reference's
normalize convention, dynamics_rk.h:42-53 and WenoLimiter.h:85-96) to the five
nonlinear WENO weights of the cell's left edge:

    x  (9)  -> a1 = W1 bf(x) + b1,  h1 = bf(relu(a1))      (32)
            -> a2 = W2 h1 + b2,     h2 = bf(relu(a2))      (32)
            -> z  = W3 h2 + b3                            (5)
            -> p  = softmax(z)

bf() rounds to bfloat16 (round to nearest even) as the tensor-core inference
does; weights enter the products rounded to bfloat16, biases stay FP32.
Training minimises the cross-entropy -sum t log p against the plain limiter's
weights t; the backward pass treats the bfloat16 roundings as identity
(straight-through) and Adam updates FP32 master weights.

Parameter vector layout (1541 floats): W1 (32x9, row major), b1 (32),
W2 (32x32), b2 (32), W3 (5x32), b3 (5).
"""
import numpy as np

N_IN, N_H, N_OUT = 9, 32, 5
SHAPES = [("W1", (N_H, N_IN)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)), ("W3", (N_OUT, N_H)),
          ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def unpack(theta):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(theta[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    return out


def pack(params):
    return np.concatenate([np.asarray(params[n], dtype=np.float64).ravel() for n, _ in SHAPES])


def normalize(s, eps=1e-20):
    """(s - min)/(max - min) per stencil; zero where the range is <= eps."""
    s = np.asarray(s, dtype=np.float32)
    mn = s.min(axis=-1, keepdims=True)
    rng = s.max(axis=-1, keepdims=True) - mn
    scale = np.where(rng > eps, rng, np.float32(1.0))
    return np.where(rng > eps, (s - mn) / scale, np.float32(0.0)).astype(np.float32)


def forward(theta, x):
    p = unpack(theta)
    W1, W2, W3 = (bf16(p[k].astype(np.float32)).astype(np.float64) for k in ("W1", "W2", "W3"))
    xb = bf16(x).astype(np.float64)
    a1 = xb @ W1.T + p["b1"]
    h1 = bf16(np.maximum(a1, 0).astype(np.float32)).astype(np.float64)
    a2 = h1 @ W2.T + p["b2"]
    h2 = bf16(np.maximum(a2, 0).astype(np.float32)).astype(np.float64)
    z = h2 @ W3.T + p["b3"]
    z = z - z.max(axis=1, keepdims=True)
    e = np.exp(z)
    prob = e / e.sum(axis=1, keepdims=True)
    return dict(xb=xb, a1=a1, h1=h1, a2=a2, h2=h2, prob=prob, W1=W1, W2=W2, W3=W3)


def loss_and_grad(theta, x, t):
    """Mean cross-entropy over the batch and its gradient (straight-through)."""
    f = forward(theta, x)
    B = x.shape[0]
    loss = -np.sum(t * np.log(np.maximum(f["prob"], 1e-30))) / B
    dz = (f["prob"] - t) / B
    g = {"W3": dz.T @ f["h2"], "b3": dz.sum(axis=0)}
    da2 = (dz @ f["W3"]) * (f["a2"] > 0)
    g["W2"] = da2.T @ f["h1"]
    g["b2"] = da2.sum(axis=0)
    da1 = (da2 @ f["W2"]) * (f["a1"] > 0)
    g["W1"] = da1.T @ f["xb"]
    g["b1"] = da1.sum(axis=0)
    return loss, pack(g)


def adam(theta, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v


def init_params(seed=0):
    """He-uniform weights, zero biases, from splitmix64 of (seed, index)."""
    idx = np.arange(N_PARAMS, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (np.uint64(seed) << np.uint64(32)) + idx + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * 2.0 - 1.0
    theta, o = np.zeros(N_PARAMS), 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        if name.startswith("W"):
            theta[o:o + n] = u[o:o + n] * np.sqrt(6.0 / shp[1])
        o += n
    return theta
