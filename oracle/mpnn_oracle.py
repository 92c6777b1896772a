"""ORACLE — test infrastructure, not product code.

numpy restatement of the learned preconditioner's network (no reference counterpart: the
network is this repository's learned preconditioner), used to check the GPU forward pass and
gradients. It follows the GPU's arithmetic where it rounds: activations h, the aggregated
messages m and the ReLU-masked gradients are rounded to BF16 where the GPU stores them in
BF16, and the layer matrices are used in BF16; everything else is FP64 (the GPU accumulates
in FP32, so agreement is to BF16-rounding level, ~1e-2 relative on gradients).

Parameter layout (FP32 vector): W_enc[64][4], b_enc[64], 3 x (W_l[64][128], b_l[64]),
w_dec[64], b_dec.
"""
from __future__ import annotations

import numpy as np

H, KIN, NF, NL = 64, 128, 4, 3
OFF_WE, OFF_BE, OFF_L0 = 0, 256, 320
LSTRIDE = 8192 + 64
OFF_WD = OFF_L0 + NL * LSTRIDE
OFF_BD = OFF_WD + 64
NPARAM = OFF_BD + 1


def bf16(a, enabled=True):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    if not enabled:
        return np.asarray(a, np.float64)
    a32 = np.ascontiguousarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, np.float64)
    p = {"We": w[OFF_WE:OFF_WE + 256].reshape(H, NF), "be": w[OFF_BE:OFF_BE + 64],
         "wd": w[OFF_WD:OFF_WD + 64], "bd": w[OFF_BD]}
    for l in range(NL):
        o = OFF_L0 + l * LSTRIDE
        p[f"W{l}"] = w[o:o + H * KIN].reshape(H, KIN)
        p[f"b{l}"] = w[o + H * KIN:o + H * KIN + H]
    return p


def graph_from_csr(row, col, val, nearwall):
    """Edges (i, j, w_ij = -a_ij / a_ii) and node features of a PPE matrix whose rows end
    with their diagonal."""
    U = len(row) - 1
    diag = val[row[1:] - 1]
    src, dst, w = [], [], []
    for i in range(U):
        for e in range(row[i], row[i + 1] - 1):
            src.append(i)
            dst.append(col[e])
            w.append(np.float32(-val[e] / diag[i]))
    deg = np.diff(row) - 1
    feat = np.stack([diag / diag.mean() - 1.0, nearwall.astype(np.float64), deg / 32.0 - 1.0], 1)
    return dict(U=U, src=np.array(src), dst=np.array(dst), w=np.array(w, np.float64),
                feat=feat.astype(np.float32).astype(np.float64), d=diag.astype(np.float32).astype(np.float64))


def apply_scaled(G, y):
    """(A D^-1 y)_i = y_i - a_ii sum_j w_ij y_j / a_jj."""
    s = np.zeros_like(y)
    np.add.at(s, G["src"], G["w"] * y[G["dst"]] / G["d"][G["dst"]])
    return y - G["d"] * s


def aggregate(G, h):
    m = np.zeros_like(h)
    np.add.at(m, G["src"], G["w"][:, None] * h[G["dst"]])
    return m


def aggregate_t(G, g):
    out = np.zeros_like(g)
    np.add.at(out, G["dst"], G["w"][:, None] * g[G["src"]])
    return out


def forward(w, G, r, round_bf16=True):
    p = unpack(w)
    U = G["U"]
    su = np.float32(np.sqrt(max(U, 1)))
    x = np.concatenate([(np.float32(r) * su).astype(np.float64)[:, None], G["feat"]], 1)
    z0 = x @ p["We"].T + p["be"]
    hs = [bf16(np.maximum(z0, 0), round_bf16)]
    zs, As = [z0], []
    for l in range(NL):
        h = hs[-1]
        m = aggregate(G, h)
        A = np.concatenate([h, bf16(m, round_bf16)], 1)
        z = A @ bf16(p[f"W{l}"], round_bf16).T + p[f"b{l}"]
        As.append(A)
        zs.append(z)
        hs.append(bf16(h + np.maximum(z, 0), round_bf16))
    y = (hs[-1] @ p["wd"] + p["bd"]) / su
    return y, dict(x=x, hs=hs, zs=zs, As=As, su=su)


def loss_and_grad(w, G, r, t, round_bf16=True, kind=0):
    """kind 0: |y - t|^2 / |t|^2; 1: |r - A D^-1 y|^2 (|r| = 1); 2: both."""
    p = unpack(w)
    y, c = forward(w, G, r, round_bf16)
    tn2 = float(np.sum(np.float64(t) ** 2))
    loss = 0.0
    gy = np.zeros_like(y)
    if kind != 1:
        loss += float(np.sum((y - t) ** 2)) / tn2
        gy += 2.0 * (y - t) / tn2
    if kind != 0:
        res = r - apply_scaled(G, y)
        loss += float(np.sum(res ** 2))
        gg = -2.0 * res
        q = np.zeros_like(y)
        np.add.at(q, G["dst"], G["d"][G["src"]] * G["w"] * gg[G["src"]])
        gy += gg - q / G["d"]
    g = np.zeros(NPARAM)
    go = gy / float(c["su"])
    g[OFF_WD:OFF_WD + 64] = c["hs"][-1].T @ go
    g[OFF_BD] = go.sum()
    gh = go[:, None] * p["wd"][None, :]
    for l in reversed(range(NL)):
        z, A = c["zs"][l + 1], c["As"][l]
        gz_f = gh * (z > 0)
        gz = bf16(gz_f, round_bf16)
        o = OFF_L0 + l * LSTRIDE
        g[o:o + H * KIN] = (gz.T @ A).ravel()
        g[o + H * KIN:o + H * KIN + H] = gz_f.sum(0)
        gA = gz @ bf16(p[f"W{l}"], round_bf16)
        gh = gh + gA[:, :H] + aggregate_t(G, gA[:, H:])
    gz0 = gh * (c["zs"][0] > 0)
    g[OFF_WE:OFF_WE + 256] = (gz0.T @ c["x"]).ravel()
    g[OFF_BE:OFF_BE + 64] = gz0.sum(0)
    return loss, g, y
