"""CPU restatement of the learned warm-start network (TEST INFRASTRUCTURE ONLY).

Mirrors csrc/mpnn.cu: inputs [b/rms(b), p/rms(p), dp/rms(dp), x, y, tag]
(dp the last pressure increment) -> encoder (6 -> 64, relu) -> 4 layers h' = relu([h | mean_j h_j | sum_j l_ij h_j] W + c) + h
-> decoder (64 -> 1); loss mean (y - t)^2.  With bf16=True the values the GPU
stores in BF16 (activations, aggregated features, layer weights) are rounded
to BF16 (round to nearest even) at the same points; the backward pass treats
those roundings as identity, as the GPU kernels do.  With bf16=False it is an
exact float64 network whose gradient is checked here by finite differences.
"""
from __future__ import annotations

import numpy as np

H, CAT, FIN, LAYERS = 64, 192, 6, 4
LAYER_PARAMS = CAT * H + H
P_WE, P_CE = 0, FIN * H
P_L0 = P_CE + H
P_WD = P_L0 + LAYERS * LAYER_PARAMS
P_CD = P_WD + H
NUM_PARAMS = P_CD + 1


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    We = P[P_WE:P_WE + FIN * H].reshape(FIN, H)
    ce = P[P_CE:P_CE + H]
    Ws, cs = [], []
    for l in range(LAYERS):
        b = P_L0 + l * LAYER_PARAMS
        Ws.append(P[b:b + CAT * H].reshape(CAT, H))
        cs.append(P[b + CAT * H:b + LAYER_PARAMS])
    return We, ce, Ws, cs, P[P_WD:P_WD + H], P[P_CD]


class Graph:
    """cloud [n][k] (row-major), lapS [n][k] = float32(lap * d_avg^2)."""

    def __init__(self, cloud, lapS):
        self.cloud = np.asarray(cloud, dtype=np.int64)
        self.w = np.asarray(lapS, dtype=np.float64)
        self.n, self.k = self.cloud.shape

    def aggregate(self, h):
        g = h[self.cloud]                       # [n][k][64]
        mean = g.sum(1) * (1.0 / self.k)
        lap = np.einsum("nk,nkf->nf", self.w, g)
        return mean, lap

    def aggregate_T(self, dmean, dlap):
        out = np.zeros((self.n, H))
        np.add.at(out, self.cloud.ravel(), np.repeat(dmean * (1.0 / self.k), self.k, axis=0))
        np.add.at(out, self.cloud.ravel(), (self.w[:, :, None] * dlap[:, None, :]).reshape(-1, H))
        return out


def forward(P, feat, G: Graph, use_bf16=True):
    We, ce, Ws, cs, wd, cd = unpack(P)
    rnd = (lambda a: bf16(a).astype(np.float64)) if use_bf16 else (lambda a: np.asarray(a, np.float64))
    feat = np.asarray(feat, np.float64)
    z0 = feat @ We + ce
    h = [rnd(np.maximum(z0, 0))]
    zs, cats = [z0], []
    for l in range(LAYERS):
        mean, lap = G.aggregate(h[-1])
        cat = np.concatenate([h[-1], rnd(mean), rnd(lap)], axis=1)
        z = cat @ rnd(Ws[l]) + cs[l]
        h.append(rnd(np.maximum(z, 0) + h[-1]))
        zs.append(z)
        cats.append(cat)
    y = h[-1] @ wd + cd
    return y, dict(h=h, z=zs, cat=cats, feat=feat)


def loss_grad(P, feat, target, G: Graph, use_bf16=True, w_mse=1.0, w_res=0.0, A=None):
    """loss = w_mse mean (y - t)^2 + w_res |A (t - y)|^2 / |A t|^2 ; A row-major [n][k] on G.cloud."""
    We, ce, Ws, cs, wd, cd = unpack(P)
    rnd = (lambda a: bf16(a).astype(np.float64)) if use_bf16 else (lambda a: np.asarray(a, np.float64))
    y, st = forward(P, feat, G, use_bf16)
    n = len(y)
    t = np.asarray(target, np.float64)
    r = y - t
    loss = w_mse * float(np.mean(r * r))
    dy = w_mse * 2 * r / n
    if w_res > 0:
        A = np.asarray(A, np.float64)
        rr = (A * (t - y)[G.cloud]).sum(1)
        q = (A * t[G.cloud]).sum(1)
        Q = float(q @ q)
        loss += w_res * float(rr @ rr) / Q
        ATr = np.zeros(n)
        np.add.at(ATr, G.cloud.ravel(), (A * rr[:, None]).ravel())
        dy = dy + w_res * (-2.0 * ATr / Q)
    g = np.zeros(NUM_PARAMS)
    h = st["h"]
    g[P_WD:P_WD + H] = h[-1].T @ dy
    g[P_CD] = dy.sum()
    dH = np.outer(dy, wd)
    for l in range(LAYERS - 1, -1, -1):
        z, cat = st["z"][l + 1], st["cat"][l]
        dz = dH * (z > 0)
        b = P_L0 + l * LAYER_PARAMS
        g[b:b + CAT * H] = (cat.T @ dz).ravel()
        g[b + CAT * H:b + LAYER_PARAMS] = dz.sum(0)
        dcat = dz @ rnd(Ws[l]).T
        dH = dH + dcat[:, :H] + G.aggregate_T(dcat[:, H:2 * H], dcat[:, 2 * H:])
    dz0 = dH * (st["z"][0] > 0)
    g[P_WE:P_WE + FIN * H] = (st["feat"].T @ dz0).ravel()
    g[P_CE:P_CE + H] = dz0.sum(0)
    return loss, g, y


def fd_check(P, feat, target, G: Graph, idx, eps=1e-6, **kw):
    """Central differences of the exact (float64) loss at parameter indices idx."""
    out = []
    for i in idx:
        Pp = np.array(P, np.float64); Pp[i] += eps
        Pm = np.array(P, np.float64); Pm[i] -= eps
        lp, _, _ = loss_grad(Pp, feat, target, G, use_bf16=False, **kw)
        lm, _, _ = loss_grad(Pm, feat, target, G, use_bf16=False, **kw)
        out.append((lp - lm) / (2 * eps))
    return np.array(out)
