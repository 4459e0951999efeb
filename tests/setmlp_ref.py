"""CPU reference of the set MLP (test infrastructure): features, forward,
mean-squared-error loss and the analytic backward, in float64, with the
weights rounded to bfloat16 as the device GEMMs use them."""
import numpy as np

F_DIM, H, O_DIM = 32, 128, 4
N_PARAM = H * F_DIM + H + H * 2 * H + H + O_DIM * H + O_DIM


def bf16(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * F_DIM].reshape(H, F_DIM); o += H * F_DIM
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * 2 * H].reshape(H, 2 * H); o += H * 2 * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + O_DIM * H].reshape(O_DIM, H); o += O_DIM * H
    b3 = p[o:o + O_DIM]
    return W1, b1, W2, b2, W3, b3


def features(inst, rmax=0.05):
    """inst: list of (N, W, H, init[N,3]) -> [sum N, 32] (float64)."""
    rows = []
    for N, W, Hh, init in inst:
        s = np.sqrt(W * Hh / N)
        c = init[:, :2]
        for i in range(N):
            d = np.sqrt(((c[i] - c) ** 2).sum(1)) + 1e-9
            d[i] = np.inf
            dd = np.sort(d)[:4]
            near = (d < 3 * s)
            w = s * s / d[near] ** 2
            vec = (c[i] - c[near]) / d[near][:, None] * w[:, None]
            rx, ry = vec.sum(0) if near.any() else (0.0, 0.0)
            f = np.zeros(F_DIM)
            x, y, r = init[i]
            f[0], f[1], f[2] = x / W, y / Hh, r / rmax
            f[3:7] = np.minimum(dd / s, 4)
            f[7], f[8], f[9], f[10] = min(x / s, 4), min((W - x) / s, 4), min(y / s, 4), min((Hh - y) / s, 4)
            f[11], f[12] = np.clip(rx * 0.25, -4, 4), np.clip(ry * 0.25, -4, 4)
            f[13], f[14] = (d < s).sum() * 0.25, (d < 2 * s).sum() * 0.1
            f[15], f[16] = N / 400, W / Hh
            f[17], f[18], f[19], f[20] = r / s, dd[0] / s - r / s, 1.0, np.sqrt(N) / 20
            rows.append(f)
    return np.array(rows)


def loss_and_grads(p, F, T, sizes):
    """F [M,32], T [M,4] (last column ignored), sizes: circles per instance."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    W1, W2, W3 = (bf16(w).astype(np.float64) for w in (W1, W2, W3))
    F = np.asarray(F, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    M = F.shape[0]
    inst = np.repeat(np.arange(len(sizes)), sizes)
    A1 = F @ W1.T + b1
    H1 = np.maximum(A1, 0)
    G = np.stack([H1[inst == b].mean(0) for b in range(len(sizes))])
    W2a, W2b = W2[:, :H], W2[:, H:]
    A2 = H1 @ W2a.T + (G @ W2b.T)[inst] + b2
    H2 = np.maximum(A2, 0)
    O = H2 @ W3.T + b3
    E = O - T
    E[:, 3] = 0
    loss = (E ** 2).sum() / (3 * M)
    dO = 2 * E / (3 * M)
    dW3 = dO.T @ H2
    db3 = dO.sum(0)
    dA2 = (dO @ W3) * (A2 > 0)
    dW2a = dA2.T @ H1
    db2 = dA2.sum(0)
    dP = np.stack([dA2[inst == b].sum(0) for b in range(len(sizes))])
    dW2b = dP.T @ G
    dG = dP @ W2b
    nb = np.array(sizes, dtype=np.float64)
    dA1 = (dA2 @ W2a + (dG / nb[:, None])[inst]) * (A1 > 0)
    dW1 = dA1.T @ F
    db1 = dA1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, np.concatenate([dW2a, dW2b], 1).ravel(), db2, dW3.ravel(), db3])
    return loss, g
