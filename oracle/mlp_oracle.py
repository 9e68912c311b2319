"""CPU oracle of the learned form's network, its training gradient and the
targets' baseline polynomial.

Test infrastructure: only the tests use this module, to check the
GPU training kernels (pmp_learn_debug_grad) and of the tensor-core inference.
There is no counterpart in the reference; the network is the project's own
surrogate (10 -> 64 -> 64 -> 64 -> 5, SiLU).

Flat parameter layout (float32, shared with the library):
  W1[64][16] (inputs 10..15 are padding)   b1[64]
  W2[64][64]                               b2[64]
  W3[64][64]                               b3[64]
  W4[8][64]  (outputs 5..7 are padding)    b4[8]
Row = output unit.  Loss = mean over rows and the 5 outputs of (y_pred - y)^2.

With quant=True the forward pass rounds weights (not biases) to bf16 (round
to nearest even) and computes each hidden activation as the inference kernel
does, silu(x) = fma(h, tanh h, h) with h = bf16(x/2), tanh h rounded to bf16
and the fma rounded once to bf16; the gradient passes through the roundings
unchanged (straight-through), as the training kernels do.
"""
import numpy as np

N_IN, N_OUT, HID = 10, 5, 64
OFF = {}
_o = 0
for _name, _size in (("W1", 64 * 16), ("b1", 64), ("W2", 64 * 64), ("b2", 64),
                     ("W3", 64 * 64), ("b3", 64), ("W4", 8 * 64), ("b4", 8)):
    OFF[_name] = (_o, _size)
    _o += _size
N_PARAM = _o
SHAPES = {"W1": (64, 16), "b1": (64,), "W2": (64, 64), "b2": (64,), "W3": (64, 64),
          "b3": (64,), "W4": (8, 64), "b4": (8,)}


def unpack(p):
    p = np.asarray(p)
    return {k: p[o:o + s].reshape(SHAPES[k]) for k, (o, s) in OFF.items()}


def pack(d):
    out = np.zeros(N_PARAM, np.float64)
    for k, (o, s) in OFF.items():
        out[o:o + s] = np.asarray(d[k], np.float64).reshape(-1)
    return out


def bf16_round(x):
    """float32 -> nearest bf16 value (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    finite = (u & 0x7F800000) != 0x7F800000
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) & 0xFFFF0000).astype(np.uint32)
    r = np.where(finite, r, u.astype(np.uint32))
    return r.view(np.float32).astype(np.float64)


def silu(h):
    return h / (1.0 + np.exp(-h))


def silu_bf16(x):
    """silu(x) with the inference kernel's bf16 roundings."""
    h = bf16_round(0.5 * np.asarray(x, np.float64))
    return bf16_round(h * bf16_round(np.tanh(h)) + h)


def dsilu(h):
    s = 1.0 / (1.0 + np.exp(-h))
    return s * (1.0 + h * (1.0 - s))


def random_params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    d = {}
    d["W1"] = np.zeros((64, 16))
    d["W1"][:, :N_IN] = rng.uniform(-1, 1, (64, N_IN)) * np.sqrt(6.0 / N_IN) * scale
    d["W2"] = rng.uniform(-1, 1, (64, 64)) * np.sqrt(6.0 / 64) * scale
    d["W3"] = rng.uniform(-1, 1, (64, 64)) * np.sqrt(6.0 / 64) * scale
    d["W4"] = np.zeros((8, 64))
    d["W4"][:N_OUT] = rng.uniform(-1, 1, (N_OUT, 64)) * np.sqrt(6.0 / 64) * scale
    for k in ("b1", "b2", "b3"):
        d[k] = rng.uniform(-0.1, 0.1, 64)
    d["b4"] = np.zeros(8)
    d["b4"][:N_OUT] = rng.uniform(-0.1, 0.1, N_OUT)
    return pack(d).astype(np.float32)


def forward(p, x, quant=False):
    """x: (n, 10) normalised inputs -> (n, 5) outputs and the saved activations."""
    w = unpack(np.asarray(p, np.float64))
    q = (lambda a: bf16_round(a)) if quant else (lambda a: a)
    act = silu_bf16 if quant else silu
    X = np.zeros((x.shape[0], 16))
    X[:, :N_IN] = x
    H1 = X @ q(w["W1"]).T + w["b1"]
    A1 = act(H1)
    H2 = A1 @ q(w["W2"]).T + w["b2"]
    A2 = act(H2)
    H3 = A2 @ q(w["W3"]).T + w["b3"]
    A3 = act(H3)
    Y = A3 @ q(w["W4"]).T + w["b4"]
    return Y[:, :N_OUT], (X, H1, A1, H2, A2, H3, A3, Y)


def loss_and_grad(p, x, y, quant=False):
    """MSE loss and its gradient with respect to the flat parameters (FP64)."""
    w = unpack(np.asarray(p, np.float64))
    q = (lambda a: bf16_round(a)) if quant else (lambda a: a)
    n = x.shape[0]
    yp, (X, H1, A1, H2, A2, H3, A3, Y) = forward(p, x, quant)
    d = yp - y
    loss = float(np.sum(d * d) / (n * N_OUT))
    dY = np.zeros((n, 8))
    dY[:, :N_OUT] = 2.0 * d / (n * N_OUT)
    g = {}
    g["W4"] = dY.T @ A3
    g["b4"] = dY.sum(0)
    dH = (dY @ q(w["W4"])) * dsilu(H3)
    g["W3"] = dH.T @ A2
    g["b3"] = dH.sum(0)
    dH = (dH @ q(w["W3"])) * dsilu(H2)
    g["W2"] = dH.T @ A1
    g["b2"] = dH.sum(0)
    dH = (dH @ q(w["W2"])) * dsilu(H1)
    g["W1"] = dH.T @ X
    g["b1"] = dH.sum(0)
    return loss, pack(g)


def infer(p, xn):
    """The inference the learned kernel runs, in FP64 apart from its roundings:
    inputs split into bf16 hi + lo, bf16 weights, the bf16 SiLU of silu_bf16,
    accumulation emulated in FP64."""
    w = unpack(np.asarray(p, np.float64))
    hi = bf16_round(xn)
    lo = bf16_round(np.asarray(xn, np.float64) - hi)
    x = hi + lo
    X = np.zeros((x.shape[0], 16))
    X[:, :N_IN] = x
    A = silu_bf16(X @ bf16_round(w["W1"]).T + w["b1"])
    A = silu_bf16(A @ bf16_round(w["W2"]).T + w["b2"])
    A = silu_bf16(A @ bf16_round(w["W3"]).T + w["b3"])
    Y = A @ bf16_round(w["W4"]).T + w["b4"]
    return Y[:, :N_OUT]


# --- the targets' baseline (learn_common.cuh base_features / learn_base,
# pmp_learn.cu solve_baseline): a polynomial in the normalised inputs whose
# residual the network predicts.  Terms, in the library's order: 1; the
# quadratic inputs z = xn[0, 1, 2, 6, 7, 8, 9]; the linear-only inputs
# xn[3, 4, 5]; ell, ell^2; g, g^2; g z_i; z_i z_j (i <= j, row by row).
BASE_Q = (0, 1, 2, 6, 7, 8, 9)
BASE_L = (3, 4, 5)
BASE_TERMS = 1 + len(BASE_Q) + len(BASE_L) + 2 + 2 + len(BASE_Q) + len(BASE_Q) * (len(BASE_Q) + 1) // 2


def base_features(xn, ell, g):
    """Terms of the baseline, float64 (rows of xn: droplets)."""
    xn = np.atleast_2d(np.asarray(xn, np.float64))
    ell = np.atleast_1d(np.asarray(ell, np.float64))
    g = np.atleast_1d(np.asarray(g, np.float64))
    z = xn[:, BASE_Q]
    cols = [np.ones(len(xn))] + [z[:, i] for i in range(z.shape[1])] + [xn[:, i] for i in BASE_L]
    cols += [ell, ell * ell, g, g * g] + [g * z[:, i] for i in range(z.shape[1])]
    cols += [z[:, i] * z[:, j] for i in range(z.shape[1]) for j in range(i, z.shape[1])]
    return np.array(cols).T


def normal_equations(F, Y):
    """The library's accumulator layout: the upper triangle of F^T F row by
    row, then F^T Y row by row."""
    G = F.T @ F
    R = F.T @ Y
    tri = np.concatenate([G[a, a:] for a in range(G.shape[0])])
    return np.concatenate([tri, R.reshape(-1)])


def solve_baseline(F, Y):
    """Ridge least squares as the library solves it: 1e-10 of each feature's
    diagonal plus 1e-14 of the largest diagonal."""
    G = F.T @ F
    d = np.diag(G).copy()
    G = G + np.diag(1e-10 * d + 1e-14 * d.max())
    return np.linalg.solve(G, F.T @ Y).T
