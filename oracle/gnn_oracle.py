"""FP64 CPU restatement of the warm-start network -- TEST INFRASTRUCTURE ONLY.

Same architecture, parameter layout, features, loss and gradient as the
engine's FP32 CUDA kernels (markov-zip1_b200/csrc/gnn.cu), written in numpy
with a hand-derived backward pass.  Tests compare the GPU loss and gradient
with this oracle, and this oracle's gradient with central finite
differences.  The network has no counterpart in the reference.
"""
from __future__ import annotations

import numpy as np

H, FV, FC = 64, 6, 5


def layout(rounds: int) -> dict:
    off, o = {}, 0

    def take(name, k):
        nonlocal o
        off[name] = (o, k)
        o += k

    take("Wve", FV * H); take("bve", H); take("Wce", FC * H); take("bce", H)
    for r in range(rounds):
        take(f"Wcs{r}", H * H); take(f"Wcn{r}", H * H); take(f"bc{r}", H)
        take(f"Wvs{r}", H * H); take(f"Wvn{r}", H * H); take(f"bv{r}", H)
    for name, k in (("wx", H), ("bx", 1), ("wy", H), ("by", 1), ("uv", H), ("uc", H), ("bw", 1)):
        take(name, k)
    off["_total"] = (o, 0)
    return off


def unpack(theta: np.ndarray, rounds: int) -> dict:
    L = layout(rounds)
    out = {}
    for k, (o, n) in L.items():
        if k == "_total":
            continue
        a = theta[o:o + n]
        if k.startswith("W"):
            a = a.reshape(-1, H)
        out[k] = a
    return out


def graph(model):
    """Dense-free graph data: CSC arrays, row/col L1 norms, features, scales."""
    m, n = model.num_rows, model.num_cols
    cs, ri, v = model.col_start, model.row_index, model.value.astype(np.float64)
    cols = np.repeat(np.arange(n), np.diff(cs))
    rn = np.zeros(m); np.add.at(rn, ri, np.abs(v))
    cn = np.zeros(n); np.add.at(cn, cols, np.abs(v))
    bs = 1.0
    for a in (model.row_lower, model.row_upper):
        f = a[np.isfinite(a)]
        if len(f):
            bs = max(bs, np.abs(f).max())
    csc = max(1.0, np.abs(model.objective).max())
    lo, hi = model.var_lower, model.var_upper
    Fv = np.stack([model.objective / csc, np.isfinite(lo), np.isfinite(hi),
                   np.where(np.isfinite(lo), np.clip(np.nan_to_num(lo, posinf=0, neginf=0) / bs, -10, 10), 0),
                   np.where(np.isfinite(hi), np.clip(np.nan_to_num(hi, posinf=0, neginf=0) / bs, -10, 10), 0),
                   cn / max(cn.max(), 1e-30)], axis=1).astype(np.float64)
    rl, ru = model.row_lower, model.row_upper
    Fc = np.stack([np.where(np.isfinite(rl), np.nan_to_num(rl, posinf=0, neginf=0) / bs, 0),
                   np.where(np.isfinite(ru), np.nan_to_num(ru, posinf=0, neginf=0) / bs, 0),
                   np.isfinite(rl), np.isfinite(ru), rn / max(rn.max(), 1e-30)], axis=1).astype(np.float64)
    rinv = np.where(rn > 0, 1.0 / np.where(rn > 0, rn, 1), 0.0)
    cinv = np.where(cn > 0, 1.0 / np.where(cn > 0, cn, 1), 0.0)
    return dict(m=m, n=n, rows=ri, cols=cols, val=v, rinv=rinv, cinv=cinv, Fv=Fv, Fc=Fc, bs=bs, cs=csc)


def _agg_c(G, hv):   # agc_i = sum_j a_ij rinv_i hv_j
    out = np.zeros((G["m"], H))
    np.add.at(out, G["rows"], (G["val"] * G["rinv"][G["rows"]])[:, None] * hv[G["cols"]])
    return out


def _agg_v(G, hc):   # agv_j = sum_i a_ij cinv_j hc_i
    out = np.zeros((G["n"], H))
    np.add.at(out, G["cols"], (G["val"] * G["cinv"][G["cols"]])[:, None] * hc[G["rows"]])
    return out


def _agg_c_t(G, d):  # d hv_j = sum_i a_ij rinv_i d_i
    out = np.zeros((G["n"], H))
    np.add.at(out, G["cols"], (G["val"] * G["rinv"][G["rows"]])[:, None] * d[G["rows"]])
    return out


def _agg_v_t(G, d):  # d hc_i = sum_j a_ij cinv_j d_j
    out = np.zeros((G["m"], H))
    np.add.at(out, G["rows"], (G["val"] * G["cinv"][G["cols"]])[:, None] * d[G["cols"]])
    return out


def relu(z):
    return np.maximum(z, 0.0)


def forward(theta, G, rounds):
    P = unpack(theta, rounds)
    hv = [relu(G["Fv"] @ P["Wve"] + P["bve"])]
    hc = [relu(G["Fc"] @ P["Wce"] + P["bce"])]
    agc, agv = [None], [None]
    for r in range(rounds):
        agc.append(_agg_c(G, hv[-1]))
        hc.append(relu(hc[-1] @ P[f"Wcs{r}"] + agc[-1] @ P[f"Wcn{r}"] + P[f"bc{r}"]))
        agv.append(_agg_v(G, hc[-1]))
        hv.append(relu(hv[-1] @ P[f"Wvs{r}"] + agv[-1] @ P[f"Wvn{r}"] + P[f"bv{r}"]))
    px = hv[-1] @ P["wx"] + P["bx"][0]
    py = hc[-1] @ P["wy"] + P["by"][0]
    lw = hv[-1].mean(0) @ P["uv"] + hc[-1].mean(0) @ P["uc"] + P["bw"][0]
    return dict(hv=hv, hc=hc, agc=agc, agv=agv, px=px, py=py, lw=lw)


def loss_and_grad(theta, model, x_target, y_target, lw_target, rounds=3):
    G = graph(model)
    F = forward(theta, G, rounds)
    P = unpack(theta, rounds)
    n, m = G["n"], G["m"]
    tx, ty = x_target / G["bs"], y_target / G["cs"]
    ex, ey, ew = F["px"] - tx, F["py"] - ty, F["lw"] - lw_target
    loss = (ex ** 2).mean() + (ey ** 2).mean() + 0.1 * ew ** 2
    g = {k: np.zeros_like(v) for k, v in P.items()}
    dx, dy, dlw = 2 * ex / n, 2 * ey / m, 0.2 * ew
    hvR, hcR = F["hv"][-1], F["hc"][-1]
    g["wx"] = dx @ hvR; g["bx"] = np.array([dx.sum()])
    g["wy"] = dy @ hcR; g["by"] = np.array([dy.sum()])
    g["uv"] = dlw * hvR.mean(0); g["uc"] = dlw * hcR.mean(0); g["bw"] = np.array([dlw])
    dhv = np.outer(dx, P["wx"]) + dlw * P["uv"] / n
    dhc = np.outer(dy, P["wy"]) + dlw * P["uc"] / m
    for r in range(rounds - 1, -1, -1):
        hv, hc = F["hv"][r + 1], F["hc"][r + 1]
        dz = dhv * (hv > 0)
        g[f"Wvs{r}"] = F["hv"][r].T @ dz; g[f"bv{r}"] = dz.sum(0); g[f"Wvn{r}"] = F["agv"][r + 1].T @ dz
        dhv_prev = dz @ P[f"Wvs{r}"].T
        dhc = dhc + _agg_v_t(G, dz @ P[f"Wvn{r}"].T)
        dzc = dhc * (hc > 0)
        g[f"Wcs{r}"] = F["hc"][r].T @ dzc; g[f"bc{r}"] = dzc.sum(0); g[f"Wcn{r}"] = F["agc"][r + 1].T @ dzc
        dhc = dzc @ P[f"Wcs{r}"].T
        dhv = dhv_prev + _agg_c_t(G, dzc @ P[f"Wcn{r}"].T)
    dz = dhv * (F["hv"][0] > 0)
    g["Wve"] = G["Fv"].T @ dz; g["bve"] = dz.sum(0)
    dz = dhc * (F["hc"][0] > 0)
    g["Wce"] = G["Fc"].T @ dz; g["bce"] = dz.sum(0)
    L = layout(rounds)
    flat = np.zeros(L["_total"][0])
    for k, (o, cnt) in L.items():
        if k != "_total":
            flat[o:o + cnt] = g[k].reshape(-1)
    return loss, flat, F


def predict(theta, model, rounds=3):
    G = graph(model)
    F = forward(theta, G, rounds)
    return F["px"] * G["bs"], F["py"] * G["cs"], F["lw"]
