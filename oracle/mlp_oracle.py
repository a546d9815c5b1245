"""CPU restatement of the surrogate MLP (test infrastructure only).

The surrogate has no counterpart in MDP; this is the project's own numpy
statement of the network the GPU kernels implement (mdp_b200/csrc/surrogate.cu):
x = (B - mu) * sinv, y = w3 . silu(W2 silu(W1 x + b1) + b2) + b3,
E = e_mu + e_sd * y, with the weight matrices rounded to BF16 (round to nearest
even) and everything else in float64.  It gives the per-atom energy, its
gradient with respect to the features, and the gradient of the training loss
mean((y - (E_ref - e_mu)/e_sd)^2) with respect to every parameter.
"""
from __future__ import annotations

import numpy as np

NK, KP, H = 14, 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * KP
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPAR = OFF_B3 + 1


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 -> nearest BF16 value (ties to even), returned as float32."""
    b = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def forward_params(P: np.ndarray) -> dict:
    """Parameters as the forward pass sees them: weights BF16-rounded, biases as is."""
    P = np.asarray(P, dtype=np.float32)
    q = P.copy()
    for a, b in ((OFF_W1, OFF_B1), (OFF_W2, OFF_B2), (OFF_W3, OFF_B3)):
        q[a:b] = bf16_round(P[a:b])
    q = q.astype(np.float64)
    return dict(W1=q[OFF_W1:OFF_B1].reshape(H, KP)[:, :NK], b1=q[OFF_B1:OFF_W2], W2=q[OFF_W2:OFF_B2].reshape(H, H),
                b2=q[OFF_B2:OFF_W3], w3=q[OFF_W3:OFF_B3], b3=q[OFF_B3])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def _silu(z):
    return z * _sig(z)


def _dsilu(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def split_norm(norm: np.ndarray):
    norm = np.asarray(norm, dtype=np.float64)
    return norm[:NK], norm[NK:2 * NK], norm[2 * NK], norm[2 * NK + 1]


def energy_and_grad(P, norm, B):
    """B (n, 14) -> per-atom energies (n,) and dE/dB (n, 14)."""
    w = forward_params(P)
    mu, sinv, emu, esd = split_norm(norm)
    x = (np.asarray(B, dtype=np.float64) - mu) * sinv
    z1 = x @ w["W1"].T + w["b1"]
    a1 = _silu(z1)
    z2 = a1 @ w["W2"].T + w["b2"]
    y = _silu(z2) @ w["w3"] + w["b3"]
    g2 = w["w3"] * _dsilu(z2)
    g1 = (g2 @ w["W2"]) * _dsilu(z1)
    gx = g1 @ w["W1"]
    return emu + esd * y, gx * sinv * esd


def loss_grad(P, norm, X, E):
    """Gradient of mean((y - t)^2), t = (E - e_mu)/e_sd, over the rows; and the loss."""
    w = forward_params(P)
    mu, sinv, emu, esd = split_norm(norm)
    x = (np.asarray(X, dtype=np.float64)[:, :NK] - mu) * sinv
    t = (np.asarray(E, dtype=np.float64) - emu) / esd
    n = x.shape[0]
    z1 = x @ w["W1"].T + w["b1"]
    a1 = _silu(z1)
    z2 = a1 @ w["W2"].T + w["b2"]
    a2 = _silu(z2)
    y = a2 @ w["w3"] + w["b3"]
    r = y - t
    dy = 2.0 * r / n
    g = np.zeros(NPAR)
    g[OFF_W3:OFF_B3] = dy @ a2
    g[OFF_B3] = dy.sum()
    d2 = dy[:, None] * w["w3"][None, :] * _dsilu(z2)
    g[OFF_W2:OFF_B2] = (d2.T @ a1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(axis=0)
    d1 = (d2 @ w["W2"]) * _dsilu(z1)
    gw1 = np.zeros((H, KP))
    gw1[:, :NK] = d1.T @ x
    g[OFF_W1:OFF_B1] = gw1.ravel()
    g[OFF_B1:OFF_W2] = d1.sum(axis=0)
    return g, float(np.mean(r * r))


def _d2silu(z):
    s = _sig(z)
    return s * (1.0 - s) * (2.0 + z * (1.0 - 2.0 * s))


def force_loss_grad(P, norm, B, db, pinfo, F_ref, E_ref, alpha, var):
    """Combined loss of the force-matching training and its parameter gradient.

    B (n, 14) features, db (npairs, 3, 14) dB_i/dr_p for pair p = (i -> j)
    (r_p = x_j - x_i), pinfo (npairs, 2) = (i, j), F_ref (n, 3), E_ref (n,).
    Loss = mean(((y - t))^2) + alpha * sum |F - F_ref|^2 / (3 n var) with
    F_a = -sum_i G_i . dB_i/dx_a and G_i = dE_i/dB_i.  Returns (grad, (Le, Lf)).
    """
    w = forward_params(P)
    mu, sinv, emu, esd = split_norm(norm)
    B = np.asarray(B, dtype=np.float64)
    n = B.shape[0]
    x = (B - mu) * sinv
    z1 = x @ w["W1"].T + w["b1"]
    a1 = _silu(z1)
    z2 = a1 @ w["W2"].T + w["b2"]
    a2 = _silu(z2)
    y = a2 @ w["w3"] + w["b3"]
    g2 = w["w3"] * _dsilu(z2)
    g1 = (g2 @ w["W2"]) * _dsilu(z1)
    G = (g1 @ w["W1"]) * sinv * esd
    i, j = pinfo[:, 0], pinfo[:, 1]
    db = np.asarray(db, dtype=np.float64)
    contrib = np.einsum("pk,pck->pc", G[i], db)
    dE = np.zeros((n, 3))
    np.add.at(dE, j, contrib)
    np.add.at(dE, i, -contrib)
    r = -dE - F_ref
    Lf = alpha * np.sum(r * r) / (3.0 * n * var)
    Q = 2.0 * alpha * r / (3.0 * n * var)
    lam = np.zeros((n, NK))
    np.add.at(lam, i, -np.einsum("pck,pc->pk", db, Q[j] - Q[i]))
    v = lam * esd * sinv
    t = (np.asarray(E_ref, dtype=np.float64) - emu) / esd
    re = y - t
    Le = float(np.mean(re * re))
    yb = 2.0 * re / n
    zd1 = v @ w["W1"].T
    ad1 = _dsilu(z1) * zd1
    zd2 = ad1 @ w["W2"].T
    ad2 = _dsilu(z2) * zd2
    g = np.zeros(NPAR)
    g[OFF_W3:OFF_B3] = yb @ a2 + ad2.sum(axis=0)
    g[OFF_B3] = yb.sum()
    z2b = yb[:, None] * w["w3"] * _dsilu(z2) + w["w3"] * _d2silu(z2) * zd2
    zd2b = w["w3"] * _dsilu(z2) * np.ones_like(z2)
    g[OFF_W2:OFF_B2] = (z2b.T @ a1 + zd2b.T @ ad1).ravel()
    g[OFF_B2:OFF_W3] = z2b.sum(axis=0)
    a1b = z2b @ w["W2"]
    ad1b = zd2b @ w["W2"]
    z1b = a1b * _dsilu(z1) + ad1b * _d2silu(z1) * zd1
    zd1b = ad1b * _dsilu(z1)
    gw1 = np.zeros((H, KP))
    gw1[:, :NK] = z1b.T @ x + zd1b.T @ v
    g[OFF_W1:OFF_B1] = gw1.ravel()
    g[OFF_B1:OFF_W2] = z1b.sum(axis=0)
    return g, (Le, Lf)
