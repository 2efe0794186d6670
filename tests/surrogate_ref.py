"""TEST INFRASTRUCTURE: a float64 numpy restatement of the surrogate network
(openifs_b200/surrogate.py) with a hand-derived backward pass, the CPU
reference the GPU kernels' gradients are checked against (and which is
itself checked against finite differences)."""
import numpy as np

LP, KLEV = 144, 137


def valid_rows(rows, lp=LP, klev=KLEV):
    pos = np.arange(rows) % lp
    return ((pos >= 2) & (pos < 2 + klev)).astype(np.float64)[:, None]


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def conv(a, w):
    """out[r] = sum_t a[r + t - T//2] @ w[t].T (zero outside)."""
    T = w.shape[0]
    rows = a.shape[0]
    out = np.zeros((rows, w.shape[1]))
    for t in range(T):
        sh = t - T // 2
        src = np.zeros_like(a)
        if sh >= 0:
            src[: rows - sh] = a[sh:]
        else:
            src[-sh:] = a[: rows + sh]
        out += src @ w[t].T
    return out


def conv_t(d, w):
    """Adjoint of conv with respect to its input."""
    T = w.shape[0]
    rows = d.shape[0]
    out = np.zeros((rows, w.shape[2]))
    for t in range(T):
        sh = t - T // 2
        contrib = d @ w[t]            # gradient w.r.t. the shifted input src
        if sh >= 0:
            out[sh:] += contrib[: rows - sh]
        else:
            out[: rows + sh] += contrib[-sh:]
    return out


def conv_w(d, a, T):
    """Gradient of sum(d * conv(a, w)) with respect to w."""
    rows = a.shape[0]
    g = np.zeros((T, d.shape[1], a.shape[1]))
    for t in range(T):
        sh = t - T // 2
        src = np.zeros_like(a)
        if sh >= 0:
            src[: rows - sh] = a[sh:]
        else:
            src[-sh:] = a[: rows + sh]
        g[t] = d.T @ src
    return g


def forward(P, x0):
    v = valid_rows(x0.shape[0])
    c = {}
    c["z1"] = (conv(x0, P["w1"]) + P["b1"]) * v
    c["h1"] = silu(c["z1"]) * v
    c["z2"] = (conv(c["h1"], P["w2"]) + P["b2"]) * v
    c["h2"] = (c["h1"] + silu(c["z2"])) * v
    c["z3"] = (conv(c["h2"], P["w3"]) + P["b3"]) * v
    c["h3"] = (c["h2"] + silu(c["z3"])) * v
    c["z4"] = (conv(c["h3"], P["w4"]) + P["b4"]) * v
    c["h4"] = silu(c["z4"]) * v
    c["y"] = (conv(c["h4"], P["w5"]) + P["b5"]) * v
    return c


def loss_and_grad(P, x0, tgt, nout=9):
    """MSE over valid rows and the first nout channels of both heads (columns
    0.. and 32..), normalised by (columns * KLEV * nout) as cs_loss does."""
    rows = x0.shape[0]
    v = valid_rows(rows)
    c = forward(P, x0)
    y = c["y"]
    count = (rows // LP) * KLEV * nout
    dy = np.zeros_like(y)
    loss = 0.0
    for h in (0, 32):
        d = (y[:, h:h + nout] - tgt[:, :nout]) * v
        loss += (d * d).sum() / count
        dy[:, h:h + nout] = 2.0 * d / count
    G = {}
    G["w5"] = conv_w(dy, c["h4"], 1)
    G["b5"] = dy.sum(0)
    dz4 = conv_t(dy, P["w5"]) * dsilu(c["z4"]) * v
    G["w4"] = conv_w(dz4, c["h3"], 1)
    G["b4"] = dz4.sum(0)
    g3 = conv_t(dz4, P["w4"]) * v
    dz3 = g3 * dsilu(c["z3"]) * v
    G["w3"] = conv_w(dz3, c["h2"], 5)
    G["b3"] = dz3.sum(0)
    g2 = (g3 + conv_t(dz3, P["w3"])) * v
    dz2 = g2 * dsilu(c["z2"]) * v
    G["w2"] = conv_w(dz2, c["h1"], 5)
    G["b2"] = dz2.sum(0)
    g1 = (g2 + conv_t(dz2, P["w2"])) * v
    dz1 = g1 * dsilu(c["z1"]) * v
    G["w1"] = conv_w(dz1, x0, 1)
    G["b1"] = dz1.sum(0)
    return loss, G


def random_params(width, rng):
    W = width
    shapes = {1: (1, W, 128), 2: (5, W, W), 3: (5, W, W), 4: (1, W, W), 5: (1, 64, W)}
    P = {}
    for i, s in shapes.items():
        P[f"w{i}"] = rng.standard_normal(s) * np.sqrt(2.0 / (s[0] * s[2])) * (0.5 if i in (2, 3) else 1.0)
        P[f"b{i}"] = rng.standard_normal(s[1]) * 0.05
    return P


def random_batch(ncol, rng):
    rows = ncol * LP
    v = valid_rows(rows)
    x0 = rng.standard_normal((rows, 128)) * v
    x0[:, 125:] = 0.0
    tgt = rng.standard_normal((rows, 16)) * v
    return x0, tgt
