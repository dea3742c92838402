"""FP32 NumPy reference of the proposal MLP (test infrastructure).

Restates what the tensor-core kernels compute, with BF16 rounding (round to nearest even)
wherever the kernels hold BF16 values: the features, the weights, the hidden activations
after bias and ReLU, and the output and hidden-layer gradients before they enter a matrix
product. Products and sums are in FP64 here (the kernels accumulate in FP32)."""
import numpy as np

SHAPES = ((64, 128), (64, 64), (64, 64), (4, 64))


def bf16(x) -> np.ndarray:
    u = np.ascontiguousarray(np.asarray(x, np.float32)).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float32)
    out, o = [], 0
    for fo, fi in SHAPES:
        W = p[o:o + fo * fi].reshape(fo, fi)
        o += fo * fi
        b = p[o:o + fo]
        o += fo
        out.append((W, b))
    return out


def pack(grads) -> np.ndarray:
    return np.concatenate([np.concatenate([dW.ravel(), db.ravel()]) for dW, db in grads]).astype(np.float64)


def _features(X):
    X = np.asarray(X, np.float32)
    Xp = np.zeros((X.shape[0], 128), np.float32)
    Xp[:, :X.shape[1]] = X
    return bf16(Xp)


def forward(p, X):
    """Logits [n][4] and the BF16 activations (input, h1, h2, h3)."""
    layers = unpack(p)
    a = _features(X)
    acts = [a]
    for k, (W, b) in enumerate(layers):
        z = acts[-1] @ bf16(W).T + b.astype(np.float64)
        if k < 3:
            acts.append(bf16(np.maximum(z.astype(np.float32), 0.0)))
        else:
            return z, acts


def loss_and_grad(p, X, labels, pos_weight=1.0):
    """Weighted logistic loss sum_{rows, outputs} w (softplus(z) - y z) / n and its gradient,
    in the parameter-block layout."""
    layers = unpack(p)
    z, acts = forward(p, X)
    n = z.shape[0]
    y = ((np.asarray(labels, np.uint8)[:, None] >> np.arange(4)) & 1).astype(np.float64)
    w = np.where(y > 0.5, pos_weight, 1.0)
    loss = float(np.sum(w * (np.logaddexp(0.0, z) - y * z)) / n)
    dz = bf16((w * (1.0 / (1.0 + np.exp(-z)) - y) / n).astype(np.float32))
    grads = [None] * 4
    for k in range(3, -1, -1):
        W, _ = layers[k]
        grads[k] = (dz.T @ acts[k], dz.sum(axis=0))
        if k > 0:
            dh = dz @ bf16(W)
            dz = bf16((dh * (acts[k] > 0)).astype(np.float32))
    return loss, pack(grads)


def _compact(v):
    v = v & 0x55555555
    v = (v | (v >> 1)) & 0x33333333
    v = (v | (v >> 2)) & 0x0F0F0F0F
    v = (v | (v >> 4)) & 0x00FF00FF
    v = (v | (v >> 8)) & 0x0000FFFF
    return v


def _dilate(v):
    v = v & 0x0000FFFF
    v = (v | (v << 8)) & 0x00FF00FF
    v = (v | (v << 4)) & 0x0F0F0F0F
    v = (v | (v << 2)) & 0x33333333
    v = (v | (v << 1)) & 0x55555555
    return v


def lvl_idx(level):
    return ((1 << (2 * level)) - 1) // 3 + 3


def proposal_features(hier, sig, L, labels_prev):
    """The proposal's feature rows (csrc/proposal_sim.cuh, k_prop_features) from a hierarchy
    (hier[field][mode]: field eta, qx, qy, z; modes 0, 1x, 1y), significance flags and the
    last step's activity bits, as BF16 values in float64: per node c of level C = L - 3, for
    the node and its eight neighbours (the centre first, then the others in row-major order
    from the south-west), h, qx, qy and z - z_centre in modes 0, 1x, 1y, scaled by 1/2, 1/4,
    1/4, 1/8 and clamped to +-16; zeros outside the mesh; then the four activity bits, 1."""
    C = L - 3
    nC = 1 << (2 * C)
    nside = 1 << C
    c = np.arange(nC, dtype=np.int64)
    x, y = _compact(c), _compact(c >> 1)
    out = np.zeros((nC, 128), np.float32)
    scale = np.float32([0.5, 0.5, 0.5, 0.25, 0.25, 0.25, 0.25, 0.25, 0.25, 0.125, 0.125, 0.125])
    order = [4, 0, 1, 2, 3, 5, 6, 7, 8]
    zc = None
    for s, k in enumerate(order):
        xx, yy = x + (k % 3) - 1, y + (k // 3) - 1
        inside = (xx >= 0) & (yy >= 0) & (xx < nside) & (yy < nside)
        code = _dilate(np.clip(xx, 0, nside - 1)) | (_dilate(np.clip(yy, 0, nside - 1)) << 1)
        lev = np.full(nC, C)
        for j in range(C - 1, -1, -1):   # the first non-significant level wins
            nonsig = sig[lvl_idx(j) + (code >> (2 * (C - j)))] == 0
            lev = np.where(nonsig, j, lev)
        node = np.array([lvl_idx(int(l)) for l in range(C + 1)])[lev] + (code >> (2 * (C - lev)))
        z0 = hier[3][0][node]
        if s == 0:
            zc = z0
        vals = []
        for m in range(3):
            vals.append(hier[0][m][node] - hier[3][m][node])
        for f in (1, 2):
            for m in range(3):
                vals.append(hier[f][m][node])
        vals += [z0 - zc, hier[3][1][node], hier[3][2][node]]
        v = np.stack([np.float32(vv) for vv in vals], axis=1).astype(np.float32) * scale
        v = np.clip(v, -16.0, 16.0)
        v[~inside] = 0.0
        out[:, 12 * s:12 * s + 12] = v
    out[:, 108:112] = (labels_prev[:, None] >> np.arange(4)) & 1
    out[:, 112] = 1.0
    return bf16(out)
