"""CPU oracle of the learned W_c frequency interpolator (test infrastructure).

The interpolator has no counterpart in the reference (the reference computes
chi0 and W at every imaginary frequency, m_llw.f90:265-376); this module is
the plain float64 statement of the network the library trains, used to check
its forward pass and its gradients:

    features  x = [v(anchor_1)/s, ..., v(anchor_na)/s, x_target, 1, 0, ...]
              s = max_a |v(anchor_a)|                         (16 features)
    output    y = C[h] . x + m_h (W3 . relu(W2^T relu(W1^T x + b1) + b2) + b3)
              m_h = 1 for head rows h < 64, 0 for the linear-only rows
    loss      L = sum_r w_r (y_r - y*_r)^2 / sum_r w_r

The MLP weights enter as their BF16 roundings (the library computes with a
BF16 copy of its FP32 master parameters); the linear head C stays FP32.
Gradients are taken with respect to the master parameters through the
rounded weights (the straight-through rule the library's Adam step uses).
The 256 x 256 layer runs on BF16 tensor-core products, so with rounding on
its operands are rounded too: the layer-1 activations h1 in the forward
pass and in the weight gradient, the layer-2 gradient g2 in the products
that give g1 and dW2 (db2 sums the unrounded g2).
"""
import numpy as np

NIN, NH, NTMAX, NMLP = 16, 256, 128, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + NIN * NH
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
OFF_C = OFF_B3 + 1
NPARAM = OFF_C + NTMAX * NIN


def bf16_round(a):
    """Round float32 values to the nearest BF16 value (ties to even)."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p, rounded=True):
    """Parameter vector -> (W1 (NIN,NH), b1, W2 (NH,NH), b2, W3, b3, C (NTMAX,NIN)) in float64.
    rounded=False keeps the given values (float64 allowed: finite differences)."""
    if rounded:
        p = np.asarray(p, dtype=np.float32)
        q = bf16_round(p)
    else:
        p = q = np.asarray(p, dtype=np.float64)
    f = lambda a: np.asarray(a, dtype=np.float64)
    return (f(q[OFF_W1:OFF_B1]).reshape(NIN, NH), f(q[OFF_B1:OFF_W2]), f(q[OFF_W2:OFF_B2]).reshape(NH, NH),
            f(q[OFF_B2:OFF_W3]), f(q[OFF_W3:OFF_B3]), float(q[OFF_B3]),
            f(p[OFF_C:]).reshape(NTMAX, NIN))


def forward(p, x, tix, rounded=True):
    """Network output for rows x (n, 16) with head rows tix (n,); returns (y, cache)."""
    W1, b1, W2, b2, W3, b3, C = unpack(p, rounded)
    x = np.asarray(x, dtype=np.float64)
    a1 = x @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    h1r = bf16_round(h1.astype(np.float32)).astype(np.float64) if rounded else h1
    a2 = h1r @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    head = np.einsum('ri,ri->r', C[tix], x)
    y = (np.asarray(tix) < NMLP) * (h2 @ W3 + b3) + head
    return y, (x, tix, h1, h2)


def loss_and_grad(p, x, tix, ystar, w=None, rounded=True):
    """Weighted MSE and its gradient with respect to the parameter vector."""
    W1, b1, W2, b2, W3, b3, C = unpack(p, rounded)
    y, (x, tix, h1, h2) = forward(p, x, tix, rounded)
    ystar = np.asarray(ystar, dtype=np.float64)
    w = np.ones_like(ystar) if w is None else np.asarray(w, dtype=np.float64)
    sw = w.sum()
    e = y - ystar
    L = float((w * e * e).sum() / sw)
    dh = 2.0 * w * e / sw                      # dL/dy
    d = dh * (np.asarray(tix) < NMLP)          # the MLP part sees only rows with an MLP term
    g = np.zeros(NPARAM, np.float64)
    g[OFF_W3:OFF_B3] = h2.T @ d
    g[OFF_B3] = d.sum()
    g2 = np.outer(d, W3) * (h2 > 0)
    if rounded:                                # the tensor-core products' BF16 operands
        h1r = bf16_round(h1.astype(np.float32)).astype(np.float64)
        g2r = bf16_round(g2.astype(np.float32)).astype(np.float64)
    else:
        h1r, g2r = h1, g2
    g[OFF_W2:OFF_B2] = (h1r.T @ g2r).ravel()
    g[OFF_B2:OFF_W3] = g2.sum(0)
    g1 = (g2r @ W2.T) * (h1 > 0)
    g[OFF_W1:OFF_B1] = (x.T @ g1).ravel()
    g[OFF_B1:OFF_W2] = g1.sum(0)
    gc = np.zeros((NTMAX, NIN))
    np.add.at(gc, tix, dh[:, None] * x)
    g[OFF_C:] = gc.ravel()
    return L, g


def features(proj, anchors, targets, thead, xcoord, rid=None, cid=None, ftab=None):
    """Samples of every (q, channel, target), target fastest.
    proj (nq, nw, ne) float32 -> x (n, 16), tix, y (normalised), w = s^2, s.
    With ftab: x[na+2..na+5] = ftab[rid[i]], ftab[cid[j]], c, [rid[i] == cid[j]]
    for channel 2 (i + nb j) + c."""
    proj = np.asarray(proj, dtype=np.float32)
    nq, nw, ne = proj.shape
    na, nt = len(anchors), len(targets)
    av = proj[:, anchors, :].transpose(0, 2, 1)            # (nq, ne, na)
    s = np.maximum(np.abs(av).max(-1), np.float32(1e-30))  # (nq, ne)
    x = np.zeros((nq, ne, nt, NIN), np.float32)
    x[..., :na] = (av / s[..., None])[:, :, None, :]
    x[..., na] = np.asarray(xcoord, np.float32)[np.asarray(targets)][None, None, :]
    x[..., na + 1] = 1.0
    if ftab is not None:
        nb = len(rid)
        e = np.arange(ne)
        i, j, c = (e >> 1) % nb, (e >> 1) // nb, e & 1
        f = np.asarray(ftab, np.float32)
        r, cc = np.asarray(rid)[i], np.asarray(cid)[j]
        x[..., na + 2] = f[r][None, :, None]
        x[..., na + 3] = f[cc][None, :, None]
        x[..., na + 4] = c[None, :, None]
        x[..., na + 5] = (r == cc)[None, :, None]
    y = proj[:, targets, :].transpose(0, 2, 1) / s[..., None]
    tix = np.broadcast_to(np.asarray(thead, np.int32)[None, None, :], (nq, ne, nt))
    ss = np.broadcast_to(s[..., None], (nq, ne, nt))
    return (x.reshape(-1, NIN), tix.reshape(-1).copy(), y.reshape(-1), (ss * ss).reshape(-1),
            ss.reshape(-1).copy())
