"""CPU oracle of the learned preconditioner's network, loss and gradient.

Test infrastructure only (the library's own kernels are what runs); plain
numpy, no automatic differentiation: the backward pass is written out by
hand so the GPU gradient is checked against an independent derivation, and
the oracle itself is checked against central finite differences.

Network (as the library's gnn.cu): width H = 64, L = 3 message-passing
layers over a graph of n nodes with K neighbour slots per node (slot 0 is
the node itself).  Inputs per node x (8), per edge e (4), aggregation weights
w (slot 0 weight 0).
    h0 = relu(W0 x + b0)
    m  = sum_slots w_is h_j ;  h(l) = relu(Ws h(l-1) + Wn m + b)
    o_is = sum_f u_f h_i,f h_j,f + c . e_is
    R = Y + O Y - T ;  loss = ||R||_F^2 / (n C)
The reference has no counterpart; parity is against this restatement.
"""
import numpy as np

FIN, EF, H, L = 8, 4, 64, 3


def n_params():
    return H * FIN + H + L * (2 * H * H + H) + H + EF


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W0 = p[o:o + H * FIN].reshape(H, FIN)
    o += H * FIN
    b0 = p[o:o + H]
    o += H
    layers = []
    for _ in range(L):
        Ws = p[o:o + H * H].reshape(H, H)
        o += H * H
        Wn = p[o:o + H * H].reshape(H, H)
        o += H * H
        b = p[o:o + H]
        o += H
        layers.append((Ws, Wn, b))
    u = p[o:o + H]
    o += H
    c = p[o:o + EF]
    o += EF
    assert o == p.size
    return W0, b0, layers, u, c


def forward(p, x, ef, w, nbr):
    """Edge outputs o[n, K] and the cache of activations."""
    W0, b0, layers, u, c = unpack(p)
    z0 = x @ W0.T + b0
    hs, zs, ms = [np.maximum(z0, 0.0)], [z0], []
    for Ws, Wn, b in layers:
        h = hs[-1]
        m = np.einsum("is,isf->if", w[:, 1:], h[nbr[:, 1:]])
        z = h @ Ws.T + m @ Wn.T + b
        ms.append(m)
        zs.append(z)
        hs.append(np.maximum(z, 0.0))
    hL = hs[-1]
    o = np.einsum("f,if,isf->is", u, hL, hL[nbr]) + ef @ c
    return o, (hs, zs, ms)


def loss_only(p, x, ef, w, nbr, Y, T):
    o, _ = forward(p, x, ef, w, nbr)
    R = Y - T + np.einsum("is,isc->ic", o, Y[nbr])
    return float((R * R).sum() / (nbr.shape[0] * Y.shape[1]))


def loss_grad(p, x, ef, w, nbr, Y, T):
    """Loss and gradient (flat, the library's parameter layout), float64."""
    W0, b0, layers, u, c = unpack(p)
    n = nbr.shape[0]
    C = Y.shape[1]
    o, (hs, zs, ms) = forward(p, x, ef, w, nbr)
    R = Y - T + np.einsum("is,isc->ic", o, Y[nbr])
    loss = float((R * R).sum() / (n * C))
    do = (2.0 / (n * C)) * np.einsum("ic,isc->is", R, Y[nbr])
    hL = hs[-1]
    gu = np.einsum("is,if,isf->f", do, hL, hL[nbr])
    gc = np.einsum("is,ise->e", do, ef)
    dh = np.einsum("is,f,isf->if", do, u, hL[nbr])
    np.add.at(dh, nbr, (do[:, :, None] * u[None, None, :]) * hL[:, None, :])
    glayers = [None] * L
    for l in range(L - 1, -1, -1):
        Ws, Wn, _ = layers[l]
        dz = dh * (zs[l + 1] > 0)
        glayers[l] = (dz.T @ hs[l], dz.T @ ms[l], dz.sum(0))
        dhp = dz @ Ws
        dm = dz @ Wn
        np.add.at(dhp, nbr[:, 1:], w[:, 1:, None] * dm[:, None, :])
        dh = dhp
    dz0 = dh * (zs[0] > 0)
    g = [(dz0.T @ x).ravel(), dz0.sum(0)]
    for gWs, gWn, gb in glayers:
        g += [gWs.ravel(), gWn.ravel(), gb]
    g += [gu, gc]
    return loss, np.concatenate(g)


def apply_precond(o, dinv, nbr, v):
    """y = (I + O) D^-1 v."""
    t = dinv * v
    return t + np.einsum("is,is->i", o, t[nbr])
