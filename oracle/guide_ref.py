"""TEST INFRASTRUCTURE: FP64 restatement of the learned guide's network.

The guide has no reference counterpart; this module is the CPU judge of the
CUDA kernels in pathtracingtutorial_b200/csrc/guide.cuh (forward of the
hash-grid + MLP + vMF mixture, and the gradient of the training loss).  Only
tests/ import it.

The model, for a position p in [0,1]^3 and a direction w:
  level l (16 levels): f = p * scale[l] + 1/2, trilinear over the 8 cell
      corners of table entries (2 features each); a corner index is
      x + y*res + z*res^2 (res = floor(scale)+2) for dense levels and
      x + (2654435761 y ^ 805459861 z) otherwise (32-bit products), modulo T;
  x = 32 features (feature 2l+f is level l, feature f);
  h1 = relu(W0 x), h2 = relu(W1 h1), h3 = relu(W2 h2), raw = W3 h3 (no biases);
  lobe k: mu = normalise(raw[5k:5k+3]), kappa = min(softplus(raw[5k+3]) + 1e-3, 5e3),
      pi = softmax(raw[5k+4 for k]);
  q(w) = sum_k pi_k kappa_k / (2 pi (1 - exp(-2 kappa_k))) exp(kappa_k (mu_k.w - 1));
  loss = mean_i  -weight_i log max(q_i(w_i), 1e-12).
Everything here is float64; the weights and grid values are the kernels' own
(BF16 / FP16 values widened to float), so the difference to the GPU is the
kernels' arithmetic only.  With bf16=True the values the kernels store as BF16
(every layer's input, and the upstream gradient entering every layer's
backward) are rounded to BF16 at the same points, which leaves only the
kernels' FP32 accumulation order and FP32 transcendentals as differences.
"""
from __future__ import annotations

import numpy as np

N_LEVELS = 16
HIDDEN = 64
OUT_PAD = 48
LOBES = 8
LAYER_SHAPES = [(HIDDEN, 2 * N_LEVELS), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (OUT_PAD, HIDDEN)]
LAYER_OFFSETS = [0, 2048, 6144, 10240]
N_WEIGHTS = 13312
P1, P2 = np.uint64(2654435761), np.uint64(805459861)


def to_bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    b = np.asarray(x, np.float64).astype(np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(weights: np.ndarray) -> list[np.ndarray]:
    w = np.asarray(weights, np.float64)
    return [w[o:o + a * b].reshape(a, b) for o, (a, b) in zip(LAYER_OFFSETS, LAYER_SHAPES)]


def _corners(params: dict, level: int, p: np.ndarray):
    """Corner table indices (n, 8) and trilinear weights (n, 8) of one level.
    The cell and its fractions are taken in float32 as the kernel does."""
    table = params["grid"].shape[1]
    s = np.float32(params["scale"][level])
    # p*s + 1/2 with one rounding (the kernel's contracted multiply-add)
    f = (p.astype(np.float32).astype(np.float64) * np.float64(s) + 0.5).astype(np.float32)
    b = np.floor(f)
    t = (f - b).astype(np.float64)
    i = b.astype(np.uint64)
    res = np.uint64(int(s) + 2)
    idx = np.empty((len(p), 8), np.int64)
    wts = np.empty((len(p), 8), np.float64)
    for c in range(8):
        cx, cy, cz = c & 1, (c >> 1) & 1, (c >> 2) & 1
        x, y, z = i[:, 0] + np.uint64(cx), i[:, 1] + np.uint64(cy), i[:, 2] + np.uint64(cz)
        if level < params["dense_limit"]:
            h = x + y * res + z * res * res
        else:
            h = x + (((y * P1) & np.uint64(0xFFFFFFFF)) ^ ((z * P2) & np.uint64(0xFFFFFFFF)))
        idx[:, c] = (h & np.uint64(table - 1)).astype(np.int64)
        wts[:, c] = (t[:, 0] if cx else 1 - t[:, 0]) * (t[:, 1] if cy else 1 - t[:, 1]) * \
                    (t[:, 2] if cz else 1 - t[:, 2])
    return idx, wts


def encode(params: dict, p: np.ndarray):
    """Encoded inputs (n, 32) and the per-level corner data for the backward."""
    grid = np.asarray(params["grid"], np.float64)
    x = np.zeros((len(p), 2 * N_LEVELS))
    corners = []
    for l in range(N_LEVELS):
        idx, wts = _corners(params, l, p)
        x[:, 2 * l:2 * l + 2] = np.einsum("nc,ncf->nf", wts, grid[l][idx])
        corners.append((idx, wts))
    return x, corners


def softplus(r):
    return np.where(r > 15, r, np.log1p(np.exp(np.minimum(r, 15))))


def mixture(raw: np.ndarray):
    """(mu (n,8,3), kappa (n,8), pi (n,8), raw mean norms (n,8), kappa clipped mask)."""
    r = raw[:, :5 * LOBES].reshape(-1, LOBES, 5)
    m = r[:, :, 0:3]
    ml = np.linalg.norm(m, axis=2)
    safe = ml > 1e-12
    mu = np.where(safe[..., None], m / np.where(safe, ml, 1)[..., None], np.array([0.0, 0.0, 1.0]))
    kraw = softplus(r[:, :, 3]) + 1e-3
    kappa = np.minimum(kraw, 5e3)
    logit = r[:, :, 4]
    e = np.exp(logit - logit.max(axis=1, keepdims=True))
    pi = e / e.sum(axis=1, keepdims=True)
    return mu, kappa, pi, np.maximum(ml, 1e-12), kraw >= 5e3


def vmf(kappa, c):
    return kappa / (2 * np.pi * -np.expm1(-2 * kappa)) * np.exp(kappa * (c - 1))


def forward(params: dict, p: np.ndarray, bf16: bool = False):
    q = to_bf16 if bf16 else (lambda a: a)
    W = layers(params["weights"])
    x, corners = encode(params, p)
    x = q(x)
    acts = [x]
    h = x
    for l in range(3):
        h = q(np.maximum(W[l] @ h.T, 0).T)
        acts.append(h)
    raw = (W[3] @ h.T).T
    return raw, acts, corners


def pdf(params: dict, p: np.ndarray, dirs: np.ndarray, bf16: bool = False) -> np.ndarray:
    raw, _, _ = forward(params, p, bf16)
    mu, kappa, pi, _, _ = mixture(raw)
    c = np.einsum("nkj,nj->nk", mu, dirs)
    return (pi * vmf(kappa, c)).sum(axis=1)


def loss(params: dict, p: np.ndarray, weight: np.ndarray, dirs: np.ndarray) -> float:
    q = pdf(params, p, np.asarray(dirs, np.float64))
    return float(np.mean(-np.asarray(weight, np.float64) * np.log(np.maximum(q, 1e-12))))


def backward(params: dict, p: np.ndarray, weight: np.ndarray, dirs: np.ndarray, bf16: bool = False):
    """Gradient of loss() with respect to the packed weights (13312,) and the
    grid (same shape as params["grid"])."""
    rq = to_bf16 if bf16 else (lambda a: a)
    p = np.asarray(p, np.float64)
    dirs = np.asarray(dirs, np.float64)
    n = len(p)
    w = np.asarray(weight, np.float64) / n
    W = layers(params["weights"])
    raw, acts, corners = forward(params, p, bf16)
    mu, kappa, pi, ml, clipped = mixture(raw)
    c = np.einsum("nkj,nj->nk", mu, dirs)
    v = vmf(kappa, c)
    q = (pi * v).sum(axis=1)
    qc = np.maximum(q, 1e-12)
    gq = -w / qc
    dr = np.zeros((n, LOBES, 5))
    # logits: d(-w log q)/d logit_k = -w pi_k (v_k / q - 1)
    dr[:, :, 4] = -w[:, None] * pi * (v / qc[:, None] - 1)
    # concentration: d log v / d kappa = 1/kappa - 2/(e^{2kappa}-1) + c - 1; d kappa / d r = sigmoid(r)
    dlogv = 1 / kappa - 2 / np.expm1(np.minimum(2 * kappa, 700)) + c - 1
    r3 = raw[:, :5 * LOBES].reshape(n, LOBES, 5)[:, :, 3]
    sig = 1 / (1 + np.exp(-r3))
    dr[:, :, 3] = np.where(clipped, 0, gq[:, None] * pi * v * dlogv * sig)
    # mean direction through the normalisation: d c / d m = (w - c mu) / |m|
    dm = (dirs[:, None, :] - c[..., None] * mu) * (gq[:, None] * pi * kappa * v / ml)[..., None]
    dr[:, :, 0:3] = dm
    d = np.zeros((n, OUT_PAD))
    d[:, :5 * LOBES] = dr.reshape(n, 5 * LOBES)
    # MLP backward
    gW = [None] * 4
    dy = rq(d)
    for l in (3, 2, 1, 0):
        gW[l] = dy.T @ acts[l]
        dx = dy @ W[l]
        if l > 0:
            dx = rq(dx * (acts[l] > 0))
        dy = dx
    gW[3][40:, :] = 0.0
    gw_flat = np.concatenate([g.ravel() for g in gW])
    # hash grid: scatter dx (n, 32) through the trilinear weights
    gg = np.zeros(params["grid"].shape, np.float64)
    for l in range(N_LEVELS):
        idx, wts = corners[l]
        for f in range(2):
            np.add.at(gg[l, :, f], idx.ravel(), (wts * dy[:, 2 * l + f:2 * l + f + 1]).ravel())
    return gw_flat, gg


def random_params(table_log2: int, seed: int, feature_scale: float = 0.3, dense_limit: int | None = None) -> dict:
    """A random network of the kernel's shape with a smaller table (for
    finite-difference checks of backward() on the CPU)."""
    rng = np.random.default_rng(seed)
    table = 1 << table_log2
    b = np.exp(np.log(2048.0 / 16.0) / (N_LEVELS - 1))
    scale = np.array([16.0 * b ** l for l in range(N_LEVELS)], np.float32)
    if dense_limit is None:
        dense_limit = 0
        for l in range(N_LEVELS):
            r = np.floor(scale[l]) + 2
            if r ** 3 <= table and dense_limit == l:
                dense_limit = l + 1
    weights = np.zeros(N_WEIGHTS)
    for l, ((a, bb), o) in enumerate(zip(LAYER_SHAPES, LAYER_OFFSETS)):
        lim = np.sqrt(6.0 / bb)
        blk = rng.uniform(-lim, lim, (a, bb))
        if l == 3:
            blk[40:] = 0.0
        weights[o:o + a * bb] = blk.ravel()
    grid = rng.uniform(-feature_scale, feature_scale, (N_LEVELS, table, 2))
    return {"weights": weights, "grid": grid, "scale": scale, "dense_limit": dense_limit,
            "lo": np.zeros(3, np.float32), "inv_extent": np.ones(3, np.float32)}
