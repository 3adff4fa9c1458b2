"""CPU oracle of the learned relay-leg proposal network.  TEST INFRASTRUCTURE ONLY.

Only the tests use this module, as the checker of the network's CUDA kernels
(forward, backward, AdamW and the tensor-core inference kernel).  The package
never imports it.

The reference has no learned proposal; what it has is the interface the network
feeds: per-shot, per-variable memory strengths for relay legs, given to the
decoder the way ``explicit_gammas`` rows are (src/pelagos/decoder.py:338-340,
481-491, 3685-3688) and clipped to ``gamma_dist_interval`` (utils.py:128-160).
This file is the network's specification, written in float64 numpy.

Network (per shot, on the Tanner graph; widths H=64 node state, D=16 message):

  features  Pc_v = clip(P_v, -1e4, 1e4)                  (P = pre-iteration posterior)
            z_v  = (tanh(Pc_v/16), [Pc_v <= 0], unsat_v, tanh(llr_v/16))
                   unsat_v = (sum of the syndrome bits of v's checks) / deg_v
            t_v  = 2*[Pc_v <= 0] + [|Pc_v| < 8]             (edge type, 0..3)
            x_c  = (s_c, mean_{v in c} z_v, 1)              (6 inputs)
  embed     q0_c = E x^_c,  g0 = relu(q0)
  layer l   m_c  = (W_l g^_c)^                              (16)
            n_v  = (sum_{c in M(v)} m_c)^
            a_c  = sum_{v in N(c)} G_l[t_v] * (n_v - m_c)  (edge-type-gated messages)
            q_c  = g_c + U_l a^_c + b_l,  g_c <- relu(q_c)  (two layers)
  readout   o_c  = O . g2^_c
            r_v  = sum_{c in M(v)} o_c / deg_v + Oz . z_v + ob
            gamma_v = lo + (hi - lo) * sigmoid(r_v)
  loss      mean over shots and variables of w_v * (softplus(r_v) - y_v r_v),
            y_v = [hard_v == e_v] (the pre-iteration decision agrees with the true
            error), w_v = 1 for y_v = 1 and w_neg otherwise.

``^`` marks the bf16 rounding the kernels apply to matrix inputs and to the
stored messages and their sums (weights are bf16; sums are float32 on the GPU,
float64 here).  With ``rounding=False`` the forward is the exact float64
function, which the finite-difference gradient check uses; gradients pass
straight through the rounding.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

H, D, F, T, XC = 64, 16, 4, 4, 6

# flat parameter layout: (name, shape), in order
LAYOUT = [("E", (H, XC)), ("W1", (D, H)), ("G1", (T, D)), ("U1", (H, D)), ("b1", (H,)),
          ("W2", (D, H)), ("G2", (T, D)), ("U2", (H, D)), ("b2", (H,)),
          ("O", (H,)), ("Oz", (F,)), ("ob", (1,))]


def offsets() -> dict:
    out, o = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = (o, shape)
        o += n
    return out


N_PARAMS = sum(int(np.prod(s)) for _, s in LAYOUT)


def unflatten(theta: np.ndarray) -> dict:
    return {k: theta[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in offsets().items()}


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest bfloat16 (ties to even), via float32."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    nan = np.isnan(f)
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(nan, np.nan, out)


@dataclass
class Graph:
    C: int
    V: int
    chk_ptr: np.ndarray   # [C+1]
    chk_var: np.ndarray   # [E] variable of each edge, check-major
    var_ptr: np.ndarray   # [V+1]
    var_chk: np.ndarray   # [E] check of each edge, variable-major (ascending checks)

    @staticmethod
    def from_csr(H_csr) -> "Graph":
        Hc = H_csr.tocsr()
        Hc.sort_indices()
        C, V = Hc.shape
        Ht = Hc.T.tocsr()
        Ht.sort_indices()
        return Graph(C, V, Hc.indptr.astype(np.int64), Hc.indices.astype(np.int64),
                     Ht.indptr.astype(np.int64), Ht.indices.astype(np.int64))

    def edge_lists(self):
        ec = np.repeat(np.arange(self.C), np.diff(self.chk_ptr))   # check of edge (check-major)
        ev = self.chk_var
        return ec, ev

    @property
    def deg_v(self):
        return np.diff(self.var_ptr)

    @property
    def deg_c(self):
        return np.diff(self.chk_ptr)


def features(g: Graph, syn: np.ndarray, post: np.ndarray, llr: np.ndarray):
    """z [B,V,4], t [B,V], x [B,C,6] (float64; x not rounded)."""
    B = syn.shape[0]
    ec, ev = g.edge_lists()
    s = syn.astype(np.float64)
    pc = np.clip(post.astype(np.float64), -1e4, 1e4)
    hard = (pc <= 0).astype(np.float64)
    degv = np.maximum(g.deg_v, 1).astype(np.float64)
    unsat = np.zeros((B, g.V))
    np.add.at(unsat.T, ev, s[:, ec].T)
    unsat /= degv
    z = np.stack([np.tanh(pc / 16), hard, unsat, np.broadcast_to(np.tanh(llr.astype(np.float64) / 16), (B, g.V))],
                 axis=2)
    t = (2 * hard + (np.abs(pc) < 8)).astype(np.int64)
    zs = np.zeros((B, g.C, F))
    np.add.at(zs.transpose(1, 0, 2), ec, z[:, ev, :].transpose(1, 0, 2))
    degc = np.maximum(g.deg_c, 1).astype(np.float64)
    x = np.concatenate([s[:, :, None], zs / degc[None, :, None], np.ones((B, g.C, 1))], axis=2)
    return z, t, x


def _gather_sum_to_vars(g: Graph, m: np.ndarray) -> np.ndarray:
    """n[b, v] = sum_{c in M(v)} m[b, c]."""
    ec, ev = g.edge_lists()
    n = np.zeros((m.shape[0], g.V) + m.shape[2:])
    np.add.at(n.swapaxes(0, 1), ev, m[:, ec].swapaxes(0, 1))
    return n


def _gather_sum_to_checks(g: Graph, x: np.ndarray) -> np.ndarray:
    """y[b, c] = sum_{v in N(c)} x[b, v]."""
    ec, ev = g.edge_lists()
    y = np.zeros((x.shape[0], g.C) + x.shape[2:])
    np.add.at(y.swapaxes(0, 1), ec, x[:, ev].swapaxes(0, 1))
    return y


def forward(theta: np.ndarray, g: Graph, syn, post, llr, rounding: bool = True, keep: bool = False):
    """Logits r [B, V] (and the saved activations when keep=True)."""
    rd = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    p = {k: rd(v) for k, v in unflatten(np.asarray(theta, np.float64)).items()}
    z, t, x = features(g, syn, post, llr)
    xr = rd(x)
    q0 = xr @ p["E"].T
    acts = {"z": z, "t": t, "xr": xr, "q0": q0}
    gprev = np.maximum(q0, 0)
    for l in (1, 2):
        W, G, U, b = p[f"W{l}"], p[f"G{l}"], p[f"U{l}"], p[f"b{l}"]
        gr = rd(gprev)
        m = rd(gr @ W.T)                                 # [B,C,D]
        n = rd(_gather_sum_to_vars(g, m))                # [B,V,D]
        Gt = G[t]                                        # [B,V,D]
        a = _gather_sum_to_checks(g, Gt * n) - _gather_sum_to_checks(g, Gt) * m
        ar = rd(a)
        q = gprev + ar @ U.T + b
        acts.update({f"gr{l}": gr, f"m{l}": m, f"n{l}": n, f"a{l}": a, f"ar{l}": ar, f"q{l}": q})
        gprev = np.maximum(q, 0)
    g2r = rd(gprev)
    o = g2r @ p["O"]                                     # [B,C]
    degv = np.maximum(g.deg_v, 1).astype(np.float64)
    r = _gather_sum_to_vars(g, o) / degv + z @ p["Oz"] + p["ob"][0]
    acts.update({"g2r": g2r, "o": o, "p": p})
    return (r, acts) if keep else r


def loss_and_dr(r: np.ndarray, y: np.ndarray, w_neg: float):
    w = np.where(y > 0, 1.0, w_neg)
    sp = np.logaddexp(0.0, r)
    L = float(np.sum(w * (sp - y * r)) / r.size)
    dr = w * (1.0 / (1.0 + np.exp(-r)) - y) / r.size
    return L, dr


def backward(theta, g: Graph, syn, post, llr, y, w_neg: float, rounding: bool = True):
    """(loss, flat gradient [N_PARAMS]) of the mean weighted logistic loss."""
    r, A = forward(theta, g, syn, post, llr, rounding=rounding, keep=True)
    L, dr = loss_and_dr(r, y.astype(np.float64), w_neg)
    p = A["p"]
    grads = {k: np.zeros_like(v) for k, v in p.items()}
    z, t = A["z"], A["t"]
    degv = np.maximum(g.deg_v, 1).astype(np.float64)
    grads["Oz"] = np.einsum("bv,bvf->f", dr, z)
    grads["ob"] = np.array([dr.sum()])
    do = _gather_sum_to_checks(g, dr / degv)             # [B,C]
    grads["O"] = np.einsum("bc,bch->h", do, A["g2r"])
    dg = do[:, :, None] * p["O"][None, None, :]          # dL/d relu(q2)
    ec, ev = g.edge_lists()
    for l in (2, 1):
        W, G, U = p[f"W{l}"], p[f"G{l}"], p[f"U{l}"]
        dq = dg * (A[f"q{l}"] > 0)
        grads[f"b{l}"] = dq.sum(axis=(0, 1))
        grads[f"U{l}"] = np.einsum("bch,bcd->hd", dq, A[f"ar{l}"])
        da = dq @ U                                      # [B,C,D]
        Gt = G[t]
        n, m = A[f"n{l}"], A[f"m{l}"]
        contrib = da[:, ec] * (n[:, ev] - m[:, ec])      # [B,E,D]: dG[t_v] += da_c (n_v - m_c)
        dG = np.zeros_like(G)
        np.add.at(dG, t[:, ev], contrib)
        grads[f"G{l}"] = dG
        dn = Gt * _gather_sum_to_vars(g, da)             # [B,V,D]
        dm = -_gather_sum_to_checks(g, Gt) * da + _gather_sum_to_checks(g, dn)
        grads[f"W{l}"] = np.einsum("bcd,bch->dh", dm, A[f"gr{l}"])
        dg = dq + dm @ W                                 # residual + message path
    dq0 = dg * (A["q0"] > 0)
    grads["E"] = np.einsum("bch,bck->hk", dq0, A["xr"])
    flat = np.concatenate([grads[k].reshape(-1) for k, _ in LAYOUT])
    return L, flat


def adamw(theta, m, v, grad, step: int, lr: float, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.01):
    """One AdamW step (decoupled weight decay, bias-corrected moments); returns new (theta, m, v)."""
    theta = theta * (1 - lr * wd)
    m = beta1 * m + (1 - beta1) * grad
    v = beta2 * v + (1 - beta2) * grad * grad
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    theta = theta - lr * mh / (np.sqrt(vh) + eps)
    return theta, m, v


def gammas(r: np.ndarray, lo: float, hi: float) -> np.ndarray:
    return lo + (hi - lo) / (1 + np.exp(-r))


def init_params(seed: int = 0) -> np.ndarray:
    """Deterministic initialisation (the network's default starting point)."""
    rng = np.random.default_rng(seed)
    p = {}
    p["E"] = rng.normal(0, 1 / np.sqrt(XC), (H, XC))
    for l in (1, 2):
        p[f"W{l}"] = rng.normal(0, 1 / np.sqrt(H), (D, H))
        p[f"G{l}"] = np.ones((T, D)) * 0.25
        p[f"U{l}"] = rng.normal(0, 0.5 / np.sqrt(D), (H, D))
        p[f"b{l}"] = np.zeros(H)
    p["O"] = rng.normal(0, 1 / np.sqrt(H), H) * 0.1
    p["Oz"] = np.array([2.0, -2.0, -1.0, 0.0])
    p["ob"] = np.array([2.0])
    return np.concatenate([p[k].reshape(-1) for k, _ in LAYOUT]).astype(np.float32)
