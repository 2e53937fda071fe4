"""Learned troubled-cell predictor on the CPU (oracle for the predictor kernels).

The predictor has no reference counterpart; this module is the plain numpy statement of
what ``csrc/mlp_kernels.cuh`` computes, used only by the tests to check those kernels:
the 8 element features (from the nodal primitive state, the P1 projector of
``hybrid/limiter.py:150-185`` and the face neighbours), the 8-64-64-64-1 ReLU/sigmoid
network, its weighted binary cross-entropy gradient and one Adam update.

Test infrastructure: only the tests use this module.
"""

import numpy as np

IN, H = 8, 64
OFF = dict(W1=0, b1=512, W2=576, b2=4672, W3=4736, b3=8832, w4=8896, b4=8960)
PARAMS = 8961


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[0:512].reshape(IN, H), w[512:576], w[576:4672].reshape(H, H), w[4672:4736],
            w[4736:8832].reshape(H, H), w[8832:8896], w[8896:8960], w[8960])


def element_stats(U, p1proj, gamma, degree=2):
    """Per element: mean rho, mean p, min/max rho, min/max p, Persson fractions of rho and p
    (0 at P1, which has no modes above the P1 space)."""
    rho = U[..., 0]
    srho = np.maximum(rho, 1e-14)
    ke = 0.5 * (U[..., 1] ** 2 + U[..., 2] ** 2 + U[..., 3] ** 2) / srho
    p = (gamma - 1.0) * (U[..., 4] - ke)
    out = np.empty((U.shape[0], 6))
    out[:, 0], out[:, 1] = rho.mean(1), p.mean(1)
    out[:, 2] = rho.min(1) / np.maximum(np.abs(rho.max(1)), 1e-30)
    out[:, 3] = p.min(1) / np.maximum(np.abs(p.max(1)), 1e-30)
    for k, m in ((4, rho), (5, p)):
        low = m @ p1proj.T
        out[:, k] = ((m - low) ** 2).sum(1) / np.maximum((m ** 2).sum(1), 1e-12) if degree >= 2 else 0.0
    return out


def features(plan, states, gamma):
    """(sum of E, 8) features in block order, from host states {etype: (E, Np, nv)}."""
    from jax_fluid_sim_b200.reference import FACE_TYPE_ID
    by_id = {FACE_TYPE_ID[k]: fp for k, fp in plan.faces.items()}
    stats = [element_stats(np.asarray(states[bp.etype]), bp.p1_projector, gamma, plan.degree) for bp in plan.blocks]
    feats = []
    for b, bp in enumerate(plan.blocks):
        st = stats[b]
        f = np.zeros((bp.E, IN))
        for e in range(bp.E):
            mr, mp = st[e, 0], st[e, 1]
            jr = jp = 0.0
            nr, npr = mr, mp
            for code in bp.elem_face[e]:
                ft, fi, side = (code >> 30) & 1, (code >> 1) & ((1 << 29) - 1), code & 1
                fp = by_id[ft]
                ob = fp.nbr_block[fi] if side == 0 else fp.owner_block[fi]
                ol = fp.nbr_local[fi] if side == 0 else fp.owner_local[fi]
                if ob < 0:
                    continue
                nb = stats[ob][ol]
                jr = max(jr, abs(nb[0] - mr) / max(abs(mr), 1e-20))
                jp = max(jp, abs(nb[1] - mp) / max(abs(mp), 1e-20))
                nr, npr = max(nr, nb[0]), max(npr, nb[1])
            f[e] = [np.log10(max(st[e, 4], 1e-12)), np.log10(max(st[e, 5], 1e-12)), jr, jp, st[e, 2], st[e, 3],
                    mr / max(nr, 1e-20), mp / max(npr, 1e-20)]
        feats.append(f)
    return np.concatenate(feats)


def forward(w, norm, X):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(w)
    x = (np.asarray(X, np.float64) - norm[:IN]) * norm[IN:]
    h1 = np.maximum(x @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    h3 = np.maximum(h2 @ W3 + b3, 0)
    z = h3 @ w4 + b4
    return 1.0 / (1.0 + np.exp(-z)), (x, h1, h2, h3)


def gradient(w, norm, X, y, pos_weight):
    """Gradient of mean_s weight_s * BCE(sigmoid(z_s), y_s), weight_s = pos_weight for y_s = 1."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(w)
    p, (x, h1, h2, h3) = forward(w, norm, X)
    y = np.asarray(y, np.float64)
    ws = np.where(y > 0.5, pos_weight, 1.0) / len(y)
    d4 = ws * (p - y)
    g = np.zeros(PARAMS)
    g[OFF["w4"]:OFF["w4"] + H] = h3.T @ d4
    g[OFF["b4"]] = d4.sum()
    d3 = np.outer(d4, w4) * (h3 > 0)
    g[OFF["W3"]:OFF["W3"] + H * H] = (h2.T @ d3).ravel()
    g[OFF["b3"]:OFF["b3"] + H] = d3.sum(0)
    d2 = (d3 @ W3.T) * (h2 > 0)
    g[OFF["W2"]:OFF["W2"] + H * H] = (h1.T @ d2).ravel()
    g[OFF["b2"]:OFF["b2"] + H] = d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    g[OFF["W1"]:OFF["W1"] + IN * H] = (x.T @ d1).ravel()
    g[OFF["b1"]:OFF["b1"] + H] = d1.sum(0)
    return g


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v
