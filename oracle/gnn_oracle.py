"""CPU FP64 restatement of the learned pressure-guess network (test
infrastructure: the checker of the library's GNN kernels, never part of the
product path).

The network has no reference counterpart (the reference starts every
pressure solve from zero, FlowSolver.inl:2203-2273); this module restates the
library's own definition (include/minicombust_gnn.h) so the device forward
and backward passes can be checked:

    h0   = relu(We x + ce),          x = [b/s_b, diag/s_d, prev/s_x, vol/mean(vol)]
    m_i  = sum_{internal slots k} (Wg e_ik + cg) * h_j
    h'   = h + W2 relu(W1 [h; m] + c1) + c2          (4 layers)
    y    = wo . relu(Wd h + cd) + co
    loss = mean((y - t/s_x - mean(y - t/s_x))^2)

`bf16=True` rounds to BF16 where the device stores BF16 (activations, GEMM
operands), so device and oracle can be compared tightly; `bf16=False` is the
plain FP64 network, whose analytic gradient is pinned by finite differences
in the tests.
"""
import numpy as np

H, L, IN = 32, 4, 4
GP_WE = 0
GP_CE = GP_WE + H * IN
GP_LAYER0 = GP_CE + H
GPL_WG, GPL_CG = 0, 2 * H
GPL_W1 = GPL_CG + H
GPL_C1 = GPL_W1 + 2 * H * H
GPL_W2 = GPL_C1 + H
GPL_C2 = GPL_W2 + H * H
GPL_SIZE = GPL_C2 + H
GP_DEC = GP_LAYER0 + L * GPL_SIZE
GPD_WD, GPD_CD = 0, H * H
GPD_WO = GPD_CD + H
GPD_CO = GPD_WO + H
NPARAM = GP_DEC + GPD_CO + 1


def bf16_round(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out = {"We": p[GP_WE:GP_WE + H * IN].reshape(H, IN), "ce": p[GP_CE:GP_CE + H], "layers": []}
    for l in range(L):
        b = GP_LAYER0 + l * GPL_SIZE
        out["layers"].append({
            "Wg": p[b + GPL_WG:b + GPL_WG + 2 * H].reshape(H, 2), "cg": p[b + GPL_CG:b + GPL_CG + H],
            "W1": p[b + GPL_W1:b + GPL_W1 + 2 * H * H].reshape(H, 2 * H), "c1": p[b + GPL_C1:b + GPL_C1 + H],
            "W2": p[b + GPL_W2:b + GPL_W2 + H * H].reshape(H, H), "c2": p[b + GPL_C2:b + GPL_C2 + H]})
    d = GP_DEC
    out["Wd"] = p[d + GPD_WD:d + GPD_WD + H * H].reshape(H, H)
    out["cd"] = p[d + GPD_CD:d + GPD_CD + H]
    out["wo"] = p[d + GPD_WO:d + GPD_WO + H]
    out["co"] = p[d + GPD_CO]
    return out


def scales(b, diag):
    b = np.asarray(b, dtype=np.float64)
    sb = np.sqrt(np.mean(b * b))
    sd = np.mean(np.asarray(diag, dtype=np.float64))
    sx = sb / sd if sd > 0 else 0.0
    if not (sb > 0 and sx > 0 and np.isfinite(sx)):
        return 0.0, 0.0, 0.0
    return sb, sd, sx


def features(graph, b, diag, prev):
    sb, sd, sx = scales(b, diag)
    rb = 1.0 / sb if sb > 0 else 0.0
    rd = 1.0 / sd if sd > 0 else 0.0
    rx = 1.0 / sx if sx > 0 else 0.0
    f32 = lambda a: np.asarray(a, dtype=np.float64).astype(np.float32).astype(np.float64)
    x = np.stack([f32(np.asarray(b, np.float64) * rb), f32(np.asarray(diag, np.float64) * rd),
                  f32(np.asarray(prev, np.float64) * rx) if prev is not None else np.zeros(len(b)),
                  np.asarray(graph["vhat"], np.float64)], axis=1)
    return x, sx


def forward(params, graph, b, diag, prev, bf16=False):
    """Returns (y, cache).  graph: dict(col [6][n] int, edge [6][n][2], vhat [n])."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    P = unpack(params)
    col = np.asarray(graph["col"])
    n = col.shape[1]
    internal = col != np.arange(n)[None, :]
    edge = np.asarray(graph["edge"], dtype=np.float64)
    x, sx = features(graph, b, diag, prev)
    h = r(np.maximum(x @ P["We"].T + P["ce"], 0.0))
    cache = {"x": x, "sx": sx, "h": [h], "u": [], "a": [], "gate": [], "internal": internal}
    for lp in P["layers"]:
        gate = edge @ lp["Wg"].T + lp["cg"]                     # [6][n][H]
        gate = np.where(internal[:, :, None], gate, 0.0)
        m = np.sum(gate * h[col], axis=0)
        u = np.concatenate([h, r(m)], axis=1)
        a = r(np.maximum(u @ r(lp["W1"]).T + lp["c1"], 0.0))
        h = r(h + (a @ r(lp["W2"]).T + lp["c2"]))
        cache["u"].append(u)
        cache["a"].append(a)
        cache["gate"].append(gate)
        cache["h"].append(h)
    q = r(np.maximum(h @ r(P["Wd"]).T + P["cd"], 0.0))
    y = q @ P["wo"] + P["co"]
    cache["q"] = q
    return y, cache


def loss_grad(params, graph, samples, bf16=False):
    """Mean loss over samples [(b, diag, prev, target)] and its gradient."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    P = unpack(params)
    col = np.asarray(graph["col"])
    n = col.shape[1]
    edge = np.asarray(graph["edge"], dtype=np.float64)
    grad = np.zeros(NPARAM)
    total = 0.0
    B = len(samples)
    for (b, diag, prev, target) in samples:
        y, c = forward(params, graph, b, diag, prev, bf16)
        sx = c["sx"]
        t = np.asarray(target, np.float64) * (1.0 / sx if sx > 0 else 0.0)
        d = y - t
        d = d - np.mean(d)
        total += np.mean(d * d)
        dy = 2.0 * d / (n * B)
        g = np.zeros(NPARAM)
        # decoder
        q, h = c["q"], c["h"][L]
        dq = np.where(q > 0, dy[:, None] * P["wo"][None, :], 0.0)
        dqr = r(dq)
        g[GP_DEC + GPD_WD:GP_DEC + GPD_WD + H * H] = (dqr.T @ h).ravel()
        g[GP_DEC + GPD_CD:GP_DEC + GPD_CD + H] = dq.sum(axis=0)
        g[GP_DEC + GPD_WO:GP_DEC + GPD_WO + H] = dy @ q
        g[GP_DEC + GPD_CO] = dy.sum()
        dh = dqr @ r(P["Wd"])
        for l in range(L - 1, -1, -1):
            lp, base = P["layers"][l], GP_LAYER0 + l * GPL_SIZE
            u, a, gate, hin = c["u"][l], c["a"][l], c["gate"][l], c["h"][l]
            dhr = r(dh)
            g[base + GPL_W2:base + GPL_W2 + H * H] = (dhr.T @ a).ravel()
            g[base + GPL_C2:base + GPL_C2 + H] = dh.sum(axis=0)
            dz = np.where(a > 0, dhr @ r(lp["W2"]), 0.0)
            dzr = r(dz)
            g[base + GPL_W1:base + GPL_W1 + 2 * H * H] = (dzr.T @ u).ravel()
            g[base + GPL_C1:base + GPL_C1 + H] = dz.sum(axis=0)
            du = dzr @ r(lp["W1"])
            dhs = dh + du[:, :H]
            dm = du[:, H:]
            # m_i = sum_k gate[k,i] * h[col[k,i]]  ->  dh[col[k,i]] += gate[k,i] * dm_i (true transpose)
            dnew = dhs.copy()
            for k in range(6):
                np.add.at(dnew, col[k], gate[k] * dm)
            contrib = dm[None, :, :] * hin[col]                 # [6][n][H], zero gate rows excluded below
            contrib = np.where(c["internal"][:, :, None], contrib, 0.0)
            g[base + GPL_WG:base + GPL_WG + 2 * H] = np.einsum("kic,kie->ce", contrib, edge).ravel()
            g[base + GPL_CG:base + GPL_CG + H] = contrib.sum(axis=(0, 1))
            dh = dnew
        dz0 = np.where(c["h"][0] > 0, dh, 0.0)
        g[GP_WE:GP_WE + H * IN] = (dz0.T @ c["x"]).ravel()
        g[GP_CE:GP_CE + H] = dz0.sum(axis=0)
        grad += g
    return total / B, grad


def graph_from_arrays(col, edge_bits, vhat):
    """Graph dict from the library's arrays (edge as packed BF16 pairs)."""
    bits = np.asarray(edge_bits, dtype=np.uint32)
    lo = (bits & 0xFFFF).astype(np.uint32) << 16
    hi = bits & 0xFFFF0000
    e = np.stack([lo.view(np.float32), hi.view(np.float32)], axis=-1).astype(np.float64)
    return {"col": np.asarray(col), "edge": e, "vhat": np.asarray(vhat, np.float64)}
