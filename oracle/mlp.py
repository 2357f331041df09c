"""CPU oracle for the learned proposal network -- TEST INFRASTRUCTURE ONLY.

Imported by tests/ as the checker of the tensor-core kernels; nothing in the
product calls it.

A numpy FP64 restatement of the network's forward and backward passes with
BF16 rounding at exactly the points where the device rounds (inputs, weights,
hidden activations, loss gradient, hidden-layer gradients), so the only
difference left is the order of the FP32 accumulations on the device:

    H_l  = bf16(relu(H_{l-1} W_l^T + b_l))          l = 1..3, H_0 = bf16(X)
    OUT  = H_3 W_4^T + b_4                          (FP32 on the device)
    loss = mean_b sum_d 0.5 ((y - mu) e^{-s})^2 + s,   s = clamp(log sigma, -7, 7)
    dOUT = bf16(dloss/dOUT)
    G_3  = bf16((dOUT W_4) * [H_3 > 0]), G_l = bf16((G_{l+1} W_{l+1}) * [H_l > 0])
    dW_l = G_l^T H_{l-1},  db_l = sum_b G_l

It also restates the spike-train features the device computes for the
network's input (log-ISI histogram, firing_rate and CV of
tools/statistics.py:15-30, spike_triggered_average of statistics.py:125-153).
"""
import numpy as np

ROWS = (512, 512, 512, 64)
COLS = (64, 512, 512, 512)


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    x = np.asarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    r = ((u + rounding) >> 16) << 16
    r = np.where(np.isnan(x), u | 0x400000, r)
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def init_params(rng, ydim=5):
    """He-style initial weights (output layer rows beyond 2*ydim zero)."""
    P = []
    for l in range(4):
        W = rng.standard_normal((ROWS[l], COLS[l])) * np.sqrt(2.0 / COLS[l])
        if l == 3:
            W *= 0.1
            W[2 * ydim:] = 0.0
        b = np.zeros(ROWS[l])
        P.append((W.astype(np.float32), b.astype(np.float32)))
    return P


def forward(P, X):
    H = [bf16(X)]
    for l in range(3):
        W, b = P[l]
        z = H[-1] @ bf16(W).T + b.astype(np.float64)
        H.append(bf16(np.maximum(z, 0.0)))
    W, b = P[3]
    out = H[-1] @ bf16(W).T + b.astype(np.float64)
    return H, out


def nll(out, Y, ydim):
    B = len(Y)
    mu = out[:, :ydim]
    sr = out[:, ydim:2 * ydim]
    s = np.clip(sr, -7.0, 7.0)
    r = (Y - mu) * np.exp(-s)
    loss = np.sum(0.5 * r * r + s) / B
    d = np.zeros((B, 64))
    d[:, :ydim] = -r * np.exp(-s) / B
    d[:, ydim:2 * ydim] = np.where((sr > -7) & (sr < 7), (1 - r * r) / B, 0.0)
    return loss, d


def gradients(P, X, Y, ydim):
    H, out = forward(P, X)
    loss, dO = nll(out, Y, ydim)
    g = bf16(dO)
    dW = [None] * 4
    db = [None] * 4
    for l in range(3, -1, -1):
        dW[l] = g.T @ H[l]
        db[l] = g.sum(axis=0)
        if l > 0:
            W = bf16(P[l][0])
            g = bf16((g @ W) * (H[l] > 0))
    return loss, dW, db, out


def features(spike_steps, stimulus, dt):
    """64 features of one train (steps) and its input (amperes)."""
    s = np.asarray(spike_steps, dtype=np.int64)
    n = len(s)
    f = np.zeros(64)
    if n >= 2:
        d = np.diff(s).astype(np.float64) * dt
        lo, hi = -3.0, np.log10(2.0)
        width = (hi - lo) / 32
        b = np.floor((np.log10(d) - lo) / width).astype(np.int64)
        b = np.clip(b, 0, 31)
        f[:32] = np.bincount(b, minlength=32)[:32] / (n - 1)
        t = s.astype(np.float64) * dt
        f[32] = (n - 1) / (t[-1] - t[0])
        f[33] = np.std(d) / np.mean(d)
        sta = np.zeros(300)
        for k in range(n):
            tk = float(s[k]) * dt
            if tk > 0.03:
                i = int(tk / dt)
                sta += np.asarray(stimulus[i - 300:i], dtype=np.float64)[::-1]
        f[34:] = sta.reshape(30, 10).sum(axis=1) / 10.0 / (n - 1) * 1e9
    return f
