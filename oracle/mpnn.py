"""ORACLE / TEST INFRASTRUCTURE ONLY.

CPU restatement (numpy) of the learned initial-partition proposal, for checking the CUDA kernels:

* features: degree, log-degree, 8 random-walk features, k -- per graph, 8 anchors by farthest-point
  sampling over hop distances (the first anchor is the lowest-id vertex of maximum degree), then the
  log-probability of a lazy random walk of T steps from each anchor landing on each vertex (T = the first
  anchor's eccentricity, at most T_MAX), standardised per graph;
* the 3-layer mean-aggregation network, layer l: Z = [H | mean over neighbours of H] @ W_l + b_l, ReLU on
  the hidden layers; BF16 weights and activations, FP32 accumulation -- the rounding points are the
  device's, so forward and backward can be compared closely;
* its backward pass and the edge-contrastive training loss on a target partition;
* the decoder: proposal coordinates P = random-walk features + the network's first 8 outputs (a residual:
  the output layer starts at zero), cut into k balanced labels by recursive inertial bisection (every part
  split at the median of its projection on its own principal axis).

Only tests/ use this module.
"""
from __future__ import annotations

import numpy as np

F_IN, HIDDEN, F_OUT = 16, 64, 16
LAYERS = [(2 * F_IN, HIDDEN), (2 * HIDDEN, HIDDEN), (2 * HIDDEN, F_OUT)]
N_ANCHORS = 8
T_MAX = 96
MARGIN = 1.0
P_FLOOR = 1e-30


def num_params() -> int:
    return sum(k * n + n for k, n in LAYERS)


def unpack(params: np.ndarray):
    out, o = [], 0
    for k, n in LAYERS:
        W = params[o:o + k * n].reshape(k, n)
        o += k * n
        b = params[o:o + n]
        o += n
        out.append((W, b))
    return out


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


def mean_agg(off, col, X):
    """Row v: mean of X over v's neighbours (0 for isolated vertices), float32 accumulation."""
    n = off.shape[0] - 1
    deg = np.diff(off)
    src = np.repeat(np.arange(n), deg)
    S = np.zeros((n, X.shape[1]), np.float32)
    np.add.at(S, src, X[col].astype(np.float32))
    inv = np.where(deg > 0, 1.0 / np.maximum(deg, 1), 0.0).astype(np.float32)
    return S * inv[:, None]


def mean_agg_t(off, col, D):
    """Transpose of mean_agg for a symmetric graph: row u gets sum over neighbours v of D[v] / deg(v)."""
    n = off.shape[0] - 1
    deg = np.diff(off)
    inv = np.where(deg > 0, 1.0 / np.maximum(deg, 1), 0.0).astype(np.float32)
    Ds = D * inv[:, None]
    src = np.repeat(np.arange(n), deg)
    out = np.zeros_like(D, dtype=np.float32)
    np.add.at(out, src, Ds[col])
    return out


# ------------------------------------------------------------------------------------------ features
def bfs(off, col, src):
    n = off.shape[0] - 1
    dist = np.full(n, -1, np.int64)
    dist[src] = 0
    front = [src]
    d = 0
    while front:
        nxt = []
        for v in front:
            for u in col[off[v]:off[v + 1]]:
                if dist[u] < 0:
                    dist[u] = d + 1
                    nxt.append(int(u))
        front = nxt
        d += 1
    return dist


def anchors(off, col):
    """Farthest-point sampling over hop distances; unreachable vertices never become anchors."""
    deg = np.diff(off)
    a = [int(np.argmax(deg))]  # argmax returns the lowest index of the maximum
    dists = [bfs(off, col, a[0])]
    ecc = int(dists[0].max())
    mind = np.where(dists[0] >= 0, dists[0], -1)
    for _ in range(1, N_ANCHORS):
        nxt = int(np.argmax(mind))  # lowest id among the farthest reachable vertices
        a.append(nxt)
        d = bfs(off, col, nxt)
        dists.append(d)
        mind = np.where(mind >= 0, np.minimum(mind, np.where(d >= 0, d, mind)), -1)
    return a, ecc


def features(off, col, k: int) -> np.ndarray:
    """Input features [n, 16] (float32, before the BF16 rounding of the network's input)."""
    n = off.shape[0] - 1
    deg = np.diff(off).astype(np.float32)
    X = np.zeros((n, F_IN), np.float32)
    if n == 0:
        return X
    mdeg = np.float32(off[-1] / n) if off[-1] > 0 else np.float32(1)
    X[:, 0] = deg / mdeg
    X[:, 1] = np.log1p(deg)
    a, ecc = anchors(off, col)
    T = min(max(ecc, 1), T_MAX)
    P = np.zeros((n, N_ANCHORS), np.float32)
    for j, s in enumerate(a):
        P[s, j] = 1.0
    inv = np.where(deg > 0, 1.0 / np.maximum(deg, 1), 0.0).astype(np.float32)
    src = np.repeat(np.arange(n), np.diff(off))
    for _ in range(T):
        Q = P * inv[:, None]
        S = np.zeros_like(P)
        np.add.at(S, src, Q[col])
        P = np.float32(0.5) * P + np.float32(0.5) * S
    L = np.log(np.maximum(P, np.float32(P_FLOOR))).astype(np.float32)
    mu = L.mean(axis=0, dtype=np.float64).astype(np.float32)
    sd = L.std(axis=0, dtype=np.float64).astype(np.float32)
    X[:, 2:2 + N_ANCHORS] = (L - mu) / np.where(sd > 0, sd, np.float32(1))
    X[:, 10] = np.float32(k) / np.float32(64)
    return X


# ------------------------------------------------------------------------------------------ network
def forward(off, col, X, params, exact: bool = False):
    """Returns (Z3 [n,16], cache).  exact=True: float64 without the BF16 roundings (for finite differences)."""
    r = (lambda x: np.asarray(x, np.float64)) if exact else bf16
    ft = np.float64 if exact else np.float32
    Ws = unpack(params)
    H = r(X)
    cache = []
    for li, (W, b) in enumerate(Ws):
        A = r(mean_agg(off, col, H.astype(ft)) if not exact else _mean64(off, col, H))
        C = np.concatenate([H, A], axis=1)
        Z = C.astype(ft) @ r(W).astype(ft) + b.astype(ft)
        cache.append((C, H))
        if li < 2:
            H = r(np.maximum(Z, 0))
        else:
            cache.append(Z)
            return Z, cache
    raise AssertionError


def _mean64(off, col, X):
    n = off.shape[0] - 1
    deg = np.diff(off)
    src = np.repeat(np.arange(n), deg)
    S = np.zeros((n, X.shape[1]), np.float64)
    np.add.at(S, src, X[col])
    return S / np.maximum(deg, 1)[:, None]


def _mean64_t(off, col, D):
    n = off.shape[0] - 1
    deg = np.diff(off)
    Ds = D / np.maximum(deg, 1)[:, None]
    src = np.repeat(np.arange(n), deg)
    out = np.zeros_like(D, dtype=np.float64)
    np.add.at(out, src, Ds[col])
    return out


def backward(off, col, cache, dZ3, params, exact: bool = False):
    """Gradients (flat) of the parameters for upstream gradient dZ3 [n,16]."""
    r = (lambda x: np.asarray(x, np.float64)) if exact else bf16
    ft = np.float64 if exact else np.float32
    Ws = unpack(params)
    grads = [None] * 3
    G = r(dZ3)
    for li in (2, 1, 0):
        C, H = cache[li]
        W, _ = Ws[li]
        dW = C.T.astype(ft) @ G.astype(ft)
        db = G.sum(axis=0, dtype=ft)
        grads[li] = (dW, db)
        if li == 0:
            break
        dC = G.astype(ft) @ r(W).T.astype(ft)
        half = dC.shape[1] // 2
        dH = dC[:, :half] + (_mean64_t(off, col, dC[:, half:]) if exact else mean_agg_t(off, col, dC[:, half:]))
        G = r(dH * (H > 0))  # H: this layer's input = the previous layer's ReLU output
    return np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads]).astype(ft)


def coords(X, Z):
    """Proposal coordinates [n,16]: random-walk features + the network's residual (first 8 outputs)."""
    P = np.zeros((X.shape[0], 16), np.float32)
    P[:, :8] = (X[:, 2:10].astype(np.float32) + Z[:, :8].astype(np.float32)).astype(np.float32)
    return P


def contrastive(off, col, Z, target):
    """Mean over arcs of y*d2 + (1-y)*max(0, MARGIN - d2), y = same target label; and dL/dZ."""
    n = off.shape[0] - 1
    src = np.repeat(np.arange(n), np.diff(off))
    diff = Z[src] - Z[col]
    d2 = (diff * diff).sum(axis=1)
    y = (target[src] == target[col])
    A = max(1, col.shape[0])
    loss = np.where(y, d2, np.maximum(0, MARGIN - d2)).sum() / A
    coef = np.where(y, 2.0, np.where(d2 < MARGIN, -2.0, 0.0)).astype(np.float32)
    g = np.zeros_like(Z, dtype=np.float32)
    np.add.at(g, src, coef[:, None] * diff)
    return np.float32(loss), (g * np.float32(2.0 / A)).astype(np.float32)


# ------------------------------------------------------------------------------------------ decoder
def orderable(x: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return np.where(u & 0x80000000, (~u) & 0xFFFFFFFF, u | 0x80000000)


def principal(P: np.ndarray, d: int = 3) -> np.ndarray:
    """Coordinates of the rows of P[:, :8] on their top-d principal axes (float64 covariance; each axis signed
    so that its largest-magnitude component is positive), as float32 [n,16] with the rest 0."""
    F = P[:, :8].astype(np.float64)
    F = F - F.mean(axis=0)
    w, V = np.linalg.eigh(F.T @ F)
    V = V[:, ::-1][:, :d]
    for j in range(d):
        if V[np.argmax(np.abs(V[:, j])), j] < 0:
            V[:, j] = -V[:, j]
    Y = np.zeros((P.shape[0], 16), np.float32)
    Y[:, :d] = (F @ V).astype(np.float32)
    return Y


def rib(P: np.ndarray, k: int) -> np.ndarray:
    """Recursive inertial bisection of the rows of P[:, :8] into k labels: every part with kp >= 2 labels
    splits at the same level into kl = kp // 2 and kp - kl labels; the left child takes the
    floor(|S| * kl / kp) vertices with the smallest (projection, id) on the part's principal axis (float64
    covariance; the axis signed so that its largest-magnitude component is positive; projection rounded to
    float32)."""
    n = P.shape[0]
    lab = np.zeros(n, np.int64)
    parts = {0: k}
    while any(kp >= 2 for kp in parts.values()):
        new = {}
        for lo, kp in parts.items():
            if kp < 2:
                new[lo] = kp
                continue
            S = np.nonzero(lab == lo)[0]
            kl = kp // 2
            nl = (len(S) * kl) // kp
            if len(S):
                F = P[S, :8].astype(np.float64)
                mu = F.mean(axis=0)
                C = (F - mu).T @ (F - mu)
                w, V = np.linalg.eigh(C)
                a = V[:, -1]
                if a[np.argmax(np.abs(a))] < 0:
                    a = -a
                y = ((F - mu) @ a).astype(np.float32)
                key = (orderable(y) << np.uint64(32)) | S.astype(np.uint64)
                order = S[np.argsort(key, kind="stable")]
                lab[order[nl:]] = lo + kl
            new[lo] = kl
            new[lo + kl] = kp - kl
        parts = new
    return lab.astype(np.int32)


def decode(X, Z, k: int) -> np.ndarray:
    return rib(coords(X, Z), k)


def rcb(Z: np.ndarray, k: int) -> np.ndarray:
    """Recursive coordinate bisection of the rows of Z into k labels.  Every part with kp >= 2 labels splits
    at the same level into kl = kp // 2 and kp - kl labels; the left child takes the floor(|S| * kl / kp)
    vertices with the smallest (coordinate, id) along the dimension of largest float32 range (lowest
    dimension on ties)."""
    n = Z.shape[0]
    Z = np.ascontiguousarray(Z, np.float32)
    lab = np.zeros(n, np.int64)
    parts = {0: k}  # lo -> number of labels
    while any(kp >= 2 for kp in parts.values()):
        new = {}
        for lo, kp in parts.items():
            if kp < 2:
                new[lo] = kp
                continue
            S = np.nonzero(lab == lo)[0]
            kl = kp // 2
            nl = (len(S) * kl) // kp
            if len(S):
                rng = (Z[S].max(axis=0) - Z[S].min(axis=0)).astype(np.float32)
                dim = int(np.argmax(rng))
                key = (orderable(Z[S, dim]) << np.uint64(32)) | S.astype(np.uint64)
                order = S[np.argsort(key, kind="stable")]
                lab[order[nl:]] = lo + kl
            new[lo] = kl
            new[lo + kl] = kp - kl
        parts = new
    return lab.astype(np.int32)
