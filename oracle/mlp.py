"""TEST INFRASTRUCTURE ONLY -- CPU restatement of the prover's proposal model.

The reference has no learned component; this module restates the model that
circlepacking_b200/csrc/cp_model.cu trains and evaluates, so that its forward
pass, loss and gradients can be checked against an independent computation.
Only tests/ and __graft_entry__.smoke() use it, as the checker.

Model (per family): 9 features -> 64 -> 64 -> 8 logits, tanh-GELU, BF16 weights
and activations as GEMM operands with FP32 (here: FP64) accumulation.
  logits 0..3  failure of sub-criterion k (binary cross-entropy, k < K)
  logits 4..7  split axis (softmax cross-entropy over the family's axes)
Features of a box (lo, hi per axis, depth): per axis d < dims the centre mapped
to [-1, 1] over the axis' nominal range and log2(max(width / range, 2^-64)) / 16
+ 1; then depth / 32.  Axis ranges: lambda [0.5, 0.99], radii [0, 0.25].
"""
from __future__ import annotations

import numpy as np

NIN, NIN_PAD, NH, NOUT = 9, 16, 64, 8
# flat parameter vector: W1 [16][64], b1 [64], W2 [64][64], b2 [64], W3 [64][8], b3 [8]
SHAPES = (("W1", (NIN_PAD, NH)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NOUT)), ("b3", (NOUT,)))
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
DIMS = (4, 3, 4, 4, 3, 4)
N_CRITERIA = (2, 1, 1, 4, 2, 2)
AXIS_RANGE = ((0.5, 0.99), (0.0, 0.25), (0.0, 0.25), (0.0, 0.25))
GELU_C = 0.7978845608028654  # sqrt(2 / pi)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def features(family: int, lo: np.ndarray, hi: np.ndarray, depth: np.ndarray) -> np.ndarray:
    """(n, 16) float32 features of boxes lo/hi (dims, n) at the given depths."""
    n = lo.shape[1]
    f = np.zeros((n, NIN_PAD), np.float64)
    for d in range(DIMS[family]):
        a, b = AXIS_RANGE[d]
        rng = b - a
        c = 0.5 * (lo[d] + hi[d])
        w = np.maximum((hi[d] - lo[d]) / rng, 2.0 ** -64)
        f[:, 2 * d] = (c - a) / rng * 2.0 - 1.0
        f[:, 2 * d + 1] = np.log2(w) / 16.0 + 1.0
    f[:, 8] = np.asarray(depth, np.float64) / 32.0
    return f.astype(np.float32)


def gelu(x):
    t = np.tanh(GELU_C * (x + 0.044715 * x ** 3))
    return 0.5 * x * (1.0 + t)


def gelu_grad(x):
    t = np.tanh(GELU_C * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C * (1.0 + 3 * 0.044715 * x * x)


def _ident(x):
    return np.asarray(x, np.float64)


def forward(p: np.ndarray, feats: np.ndarray, exact: bool = False) -> dict:
    """exact=True skips every BF16 rounding (for finite-difference checks)."""
    bf16 = _ident if exact else globals()["bf16"]
    w = unpack(np.asarray(p, np.float64 if exact else np.float32))
    x = bf16(feats)
    h1 = x @ bf16(w["W1"]) + w["b1"]
    g1 = bf16(gelu(h1))
    h2 = g1 @ bf16(w["W2"]) + w["b2"]
    g2 = bf16(gelu(h2))
    z = g2 @ bf16(w["W3"]) + w["b3"]
    return dict(x=x, h1=h1, g1=g1, h2=h2, g2=g2, z=z)


def loss_grad(family: int, p: np.ndarray, feats: np.ndarray, crit: np.ndarray, axis: np.ndarray, exact: bool = False):
    """Mean loss over the rows and its gradient with respect to the flat parameters.

    crit: uint8 failure bits per row (bit k = sub-criterion k fails);
    axis: int8 best split axis per row, -1 = no label."""
    K, D = min(N_CRITERIA[family], 4), DIMS[family]
    bf16 = _ident if exact else globals()["bf16"]
    w = unpack(np.asarray(p, np.float64 if exact else np.float32))
    f = forward(p, feats, exact)
    z = f["z"]
    B = z.shape[0]
    y = ((crit[:, None].astype(np.int64) >> np.arange(4)) & 1).astype(np.float64)
    zc = z[:, :K]
    loss = (np.logaddexp(0.0, zc) - y[:, :K] * zc).sum()
    dz = np.zeros_like(z)
    dz[:, :K] = 1.0 / (1.0 + np.exp(-zc)) - y[:, :K]
    has = axis >= 0
    za = z[:, 4:4 + D]
    m = za.max(axis=1, keepdims=True)
    e = np.exp(za - m)
    sm = e / e.sum(axis=1, keepdims=True)
    lse = (m[:, 0] + np.log(e.sum(axis=1)))
    ai = np.where(has, axis, 0).astype(np.int64)
    loss += (np.where(has, lse - za[np.arange(B), ai], 0.0)).sum()
    onehot = np.zeros_like(za)
    onehot[np.arange(B), ai] = 1.0
    dz[:, 4:4 + D] = np.where(has[:, None], sm - onehot, 0.0)
    loss /= B
    dz /= B
    dzb = bf16(dz)
    g = {}
    g["W3"] = f["g2"].T @ dzb
    g["b3"] = dz.sum(axis=0)
    dg2 = dzb @ bf16(w["W3"]).T
    dh2 = dg2 * gelu_grad(f["h2"])
    dh2b = bf16(dh2)
    g["W2"] = f["g1"].T @ dh2b
    g["b2"] = dh2.sum(axis=0)
    dg1 = dh2b @ bf16(w["W2"]).T
    dh1 = dg1 * gelu_grad(f["h1"])
    dh1b = bf16(dh1)
    g["W1"] = f["x"].T @ dh1b
    g["b1"] = dh1.sum(axis=0)
    flat = np.concatenate([g[name].reshape(-1) for name, _ in SHAPES])
    return float(loss), flat


def init_params(seed: int) -> np.ndarray:
    """Deterministic initialisation (uniform +-1/sqrt(fan_in)), padded input rows zero."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in SHAPES:
        fan_in = NIN if name in ("W1", "b1") else NH
        a = rng.uniform(-1.0, 1.0, shape) / np.sqrt(fan_in)
        if name == "W1":
            a[NIN:] = 0.0
        parts.append(a.reshape(-1))
    return np.concatenate(parts).astype(np.float32)
