"""Test infrastructure (the oracle), not part of the product: a numpy restatement of the troubled-cell sensor's inputs,
labels and network, the check of the GPU sensor kernels (fenice_b200/csrc/sensor.cuh).

* scales(Q5): the physical scale of each quantity at the centre cell: rho, the sound speed sqrt(gamma (p + p_inf) / rho)
  for the three velocities, p + p_inf (rho and p + p_inf at least 1e-30).
* stencil_features(Q5): the 25 features of one (cell, axis): the 5 cells c-2 .. c+2 along the axis, 5 primitive
  quantities each (rho, normal velocity, the two tangential velocities (0 on a 2-D mesh), p). Per quantity, with
  M = max_k |v_k - v0| and s its scale: the shape (v_k - v0) / M of the four neighbours (0 when M = 0) times
  min(1, 1e4 M / s) and, in the centre slot, the amplitude log2(1 + 1e4 M / s) / 4; quantity-major, padded with zeros to
  32 inputs.
* departure(Q5): the label statistic: over the 5 quantities and both WENO5-Z reconstructions centred on the cell (the
  value at its right face from c-2 .. c+2 and at its left face from c+2 .. c-2), the largest gap between the WENO5-Z
  value (the reference's weno5z, cpp/src/Schemes.cpp:328-353) and the linear fifth-order upwind value
  (2 c0 - 13 c1 + 47 c2 + 27 c3 - 3 c4) / 60, relative to the quantity's scale. A cell is troubled along the axis when it
  exceeds the label threshold.
* mlp_forward / mlp_loss_grad: 32 -> 32 -> 32 -> 1 with ReLU, the product's arithmetic emulated: inputs, weights and
  hidden activations rounded to bfloat16 where the kernels feed them to the tensor cores, sums and biases in float32 (here
  float64 on the rounded operands), loss the mean class-weighted binary cross-entropy with logits.
* gate_tiles: the stage tiles' gate from the network's flags of every (cell, axis): the troubled set grown by the travel
  radius, then reduced to the tiles (stated below as two separate steps; the device does both in one pass).
"""
import numpy as np

D_LIN = np.array([0.1, 0.6, 0.3])
NF, NK, NH = 25, 32, 32


def bf16(a):
    """Round to bfloat16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def axis_quantities(W, axis):
    """(..., 5, 5) stencil of primitive cells [rho, u, v, p, w] along `axis` -> [rho, u_n, u_t1, u_t2, p]."""
    W = np.asarray(W, dtype=np.float64)
    u, v, w = W[..., 1], W[..., 2], W[..., 4]
    n, t1, t2 = [(u, v, w), (v, w, u), (w, u, v)][axis]
    return np.stack([W[..., 0], n, t1, t2, W[..., 3]], axis=-1)


def scales(Q5, gamma=1.4, p_inf=0.0):
    """(n, 5, 5) stencil quantities -> (n, 5) physical scale of each quantity at the centre cell."""
    Q5 = np.asarray(Q5, dtype=np.float64)
    rho = np.maximum(Q5[:, 2, 0], 1e-30)
    pp = np.maximum(Q5[:, 2, 4] + p_inf, 1e-30)
    c = np.sqrt(gamma * pp / rho)
    return np.stack([rho, c, c, c, pp], axis=1)


def stencil_features(Q5, gamma=1.4, p_inf=0.0):
    """(n, 5, 5) stencil quantities -> (n, 32) features (quantity-major: 5 entries per quantity, positions c-2 .. c+2
    with the amplitude in the centre entry; columns 25 .. 31 zero)."""
    sc = scales(Q5, gamma, p_inf).astype(np.float32)
    Q5 = np.asarray(Q5, dtype=np.float32)
    d = Q5 - Q5[:, 2:3, :]
    M = np.abs(d).max(axis=1)
    a = (np.float32(1e4) * M / sc).astype(np.float32)
    g = np.minimum(np.float32(1.0), a)
    iM = np.where(M > 0, g / np.where(M > 0, M, 1), 0).astype(np.float32)
    f = d * iM[:, None, :]
    f[:, 2, :] = 0.25 * np.log2(1.0 + a)
    out = np.zeros((len(Q5), NK), dtype=np.float32)
    out[:, :NF] = np.transpose(f, (0, 2, 1)).reshape(len(Q5), NF)
    return out


def weno5z_weights(c, eps_rel=1e-6):
    """WENO-Z weights of the value at the face right of c[:, 2] from c[:, 0..4] (float64)."""
    c0, c1, c2, c3, c4 = (c[:, k] for k in range(5))
    eps = eps_rel * (c0 * c0 + c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4) * 0.2 + 1e-300
    s0, t0 = c0 - 2 * c1 + c2, c0 - 4 * c1 + 3 * c2
    s1, t1 = c1 - 2 * c2 + c3, c1 - c3
    s2, t2 = c2 - 2 * c3 + c4, 3 * c2 - 4 * c3 + c4
    b0 = 13 / 12 * s0 * s0 + 0.25 * t0 * t0
    b1 = 13 / 12 * s1 * s1 + 0.25 * t1 * t1
    b2 = 13 / 12 * s2 * s2 + 0.25 * t2 * t2
    tau = np.abs(b0 - b2)
    a = np.stack([0.1 * (1 + tau / (b0 + eps)), 0.6 * (1 + tau / (b1 + eps)), 0.3 * (1 + tau / (b2 + eps))], axis=1)
    return a / a.sum(axis=1, keepdims=True)


def weno5z_value(c, eps_rel=1e-6):
    """The WENO5-Z value at the face right of c[:, 2] from c[:, 0..4] (float64, the operation order of the reference's
    weno5z, cpp/src/Schemes.cpp:341-353)."""
    c0, c1, c2, c3, c4 = (c[:, k] for k in range(5))
    eps = eps_rel * (c0 * c0 + c1 * c1 + c2 * c2 + c3 * c3 + c4 * c4) * 0.2 + 1e-300
    p0 = (2 * c0 - 7 * c1 + 11 * c2) / 6
    p1 = (-c1 + 5 * c2 + 2 * c3) / 6
    p2 = (2 * c2 + 5 * c3 - c4) / 6
    s0, t0 = c0 - 2 * c1 + c2, c0 - 4 * c1 + 3 * c2
    s1, t1 = c1 - 2 * c2 + c3, c1 - c3
    s2, t2 = c2 - 2 * c3 + c4, 3 * c2 - 4 * c3 + c4
    b0 = 13 / 12 * s0 * s0 + 0.25 * t0 * t0
    b1 = 13 / 12 * s1 * s1 + 0.25 * t1 * t1
    b2 = 13 / 12 * s2 * s2 + 0.25 * t2 * t2
    tau = np.abs(b0 - b2)
    a0, a1, a2 = 0.1 * (1 + tau / (b0 + eps)), 0.6 * (1 + tau / (b1 + eps)), 0.3 * (1 + tau / (b2 + eps))
    return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2)


def linear_value(c):
    """The linear fifth-order upwind value at the face right of c[:, 2]."""
    return (2 * c[:, 0] - 13 * c[:, 1] + 47 * c[:, 2] + 27 * c[:, 3] - 3 * c[:, 4]) / 60


def departure(Q5, eps_rel=1e-6, gamma=1.4, p_inf=0.0):
    """(n, 5, 5) -> (n,) the largest |WENO5-Z - linear| face-value gap relative to the quantity's scale."""
    Q5 = np.asarray(Q5, dtype=np.float64)
    sc = scales(Q5, gamma, p_inf)
    out = np.zeros(len(Q5))
    for q in range(Q5.shape[2]):
        c = Q5[:, :, q]
        for cc in (c, c[:, ::-1]):
            out = np.maximum(out, np.abs(weno5z_value(cc, eps_rel) - linear_value(cc)) / sc[:, q])
    return out


def mlp_forward(X, P):
    """Logits of (n, 32) features; P = dict(W1 (32, 32), b1 (32,), W2 (32, 32), b2, w3 (32,), b3 ()). Returns the
    logits and the intermediates mlp_backward needs."""
    Xb = bf16(X).astype(np.float64)
    W1, W2, w3 = (bf16(P[k]).astype(np.float64) for k in ("W1", "W2", "w3"))
    z1 = Xb @ W1.T + P["b1"]
    h1 = bf16(np.maximum(z1, 0)).astype(np.float64)
    z2 = h1 @ W2.T + P["b2"]
    h2 = bf16(np.maximum(z2, 0)).astype(np.float64)
    z = h2 @ w3 + float(P["b3"])
    return z, (Xb, z1, h1, z2, h2, W1, W2, w3)


def mlp_loss_grad(X, y, wpos, P):
    """Mean class-weighted BCE with logits (weight wpos on y = 1, 1 on y = 0) and its gradients. The backward pass
    rounds the back-propagated hidden gradients to bfloat16 where the kernels do (before the weight-gradient and
    input-gradient products)."""
    z, (Xb, z1, h1, z2, h2, W1, W2, w3) = mlp_forward(X, P)
    n = len(z)
    y = np.asarray(y, dtype=np.float64)
    w = np.where(y > 0.5, wpos, 1.0)
    sp = np.logaddexp(0, -np.abs(z)) + np.maximum(z, 0)   # softplus(z)
    loss = float(np.mean(w * (sp - y * z)))
    dz = w * (1 / (1 + np.exp(-z)) - y) / n
    G = {"w3": h2.T @ dz, "b3": dz.sum()}
    dh2 = np.outer(dz, w3) * (z2 > 0)
    dh2b = bf16(dh2).astype(np.float64)
    G["W2"] = dh2b.T @ h1
    G["b2"] = dh2.sum(axis=0)
    dh1 = (dh2b @ W2) * (z1 > 0)
    dh1b = bf16(dh1).astype(np.float64)
    G["W1"] = dh1b.T @ Xb
    G["b1"] = dh1.sum(axis=0)
    return loss, G


def gate_tiles(cell_flags, tile, radius, periodic):
    """The gate of the stage tiles from the network's flags (cell_flags: (dim, nz, ny, nx), 1 = the cell's
    reconstructions along that axis stay WENO5-Z). (1) Every axis plane grown by `radius` cells along each mesh axis, one
    axis after the other: a cell is flagged when a flagged cell lies within `radius` along that axis, the index wrapped
    across a periodic pair of sides and dropped beyond the others. (2) Per axis a and tile (tile = cells per axis, the
    last tile cut at the mesh end): 1 when a flagged cell lies in the tile extended by one cell along a (wrapped across a
    periodic side), or when that extension leaves the mesh across a side that is not periodic. Returns
    (dim, tiles z, tiles y, tiles x) uint8."""
    f = np.asarray(cell_flags).astype(bool)
    dim = f.shape[0]
    n3 = (f.shape[3], f.shape[2], f.shape[1])
    for d in range(dim):
        ax = 3 - d   # mesh axis d is numpy axis 3 - d of (dim, nz, ny, nx)
        g = np.zeros_like(f)
        for o in range(-radius, radius + 1):
            if periodic[d]:
                g |= np.roll(f, -o, axis=ax)   # g[i] |= f[(i + o) mod n]
            else:
                src = [slice(None)] * 4
                dst = [slice(None)] * 4
                n = n3[d]
                if o >= 0:
                    src[ax], dst[ax] = slice(o, n), slice(0, max(n - o, 0))
                else:
                    src[ax], dst[ax] = slice(0, max(n + o, 0)), slice(-o, n)
                g[tuple(dst)] |= f[tuple(src)]
        f = g
    tiles = [(n3[d] + tile[d] - 1) // tile[d] for d in range(3)]
    out = np.zeros((dim, tiles[2], tiles[1], tiles[0]), dtype=np.uint8)
    for a in range(dim):
        for t2 in range(tiles[2]):
            for t1 in range(tiles[1]):
                for t0 in range(tiles[0]):
                    o = (t0 * tile[0], t1 * tile[1], t2 * tile[2])
                    lo = list(o)
                    hi = [min(o[d] + tile[d] - 1, n3[d] - 1) for d in range(3)]
                    lo[a] -= 1
                    hi[a] += 1
                    if not periodic[a] and (lo[a] < 0 or hi[a] > n3[a] - 1):
                        out[a, t2, t1, t0] = 1
                        continue
                    idx = [np.arange(lo[d], hi[d] + 1) % n3[d] for d in range(3)]
                    out[a, t2, t1, t0] = f[a][np.ix_(idx[2], idx[1], idx[0])].any()
    return out
