"""CPU oracle of the learned preconditioner (test infrastructure only).

The learned preconditioner has no counterpart in the reference (CICY_geom
always runs Jacobi-PCG, Direct_Electrifying.cpp:1538-1735).  This module
restates, in numpy, exactly what the device kernels in
cicy_geom_b200/csrc/learned.cu compute, so the tests can check the device
forward pass and gradients against it:

  features   node: ((log d_i - mean) / std, log(1 + deg_i));
             entry (i, k): lc = log|a_ik| - (log d_i + log d_k) / 2, jf = 1 for a
             tunnelling junction (not two consecutive nodes of one CNT chain)
  layer 0    H = bf16(relu(f W_in + b_in))                       (width 32)
  layers 1-3 G = bf16(H U_l); gate_ik = sigmoid(p0 lc + p1 jf + p2)
             M_i = (1/deg_i) sum_k gate_ik G_k; A = H W_l + M + b_l
             H = bf16(H + relu(A))
  edge out   o_ik = sum_j v_j H_ij H_kj + q0 lc_ik + q1; w_ik = sigmoid(o_ik)
  precond    T = chain blocks (consecutive free nodes of one CNT, split every
             32 rows; a singular block falls back to its diagonal),
             E_w = w_ik |a_ik| on the couplings outside T;
             z = y + T^-1 (E_w y),  y = T^-1 r
  loss       per probe u: r = A u, q = A z, L = 1 - (r.q)^2 / (|r|^2 |q|^2)
             (one minus the squared cosine: the residual left by one
             optimally scaled preconditioned Richardson step), averaged.

bf16() rounds float32 to bfloat16 (round to nearest even) at the points where
the device stores BF16; the backward pass treats the rounding as identity.
With rounding=False everything is float64, for finite-difference checks.
"""
from __future__ import annotations

import numpy as np

WIDTH = 32
LAYERS = 3
BLOCK_MAX = 32


def layout():
    """(name, shape) of each parameter, in the order of the flat vector."""
    out = [("W_in", (2, WIDTH)), ("b_in", (WIDTH,))]
    for l in range(LAYERS):
        out += [(f"U{l}", (WIDTH, WIDTH)), (f"W{l}", (WIDTH, WIDTH)), (f"b{l}", (WIDTH,)), (f"p{l}", (3,))]
    out += [("v", (WIDTH,)), ("q", (2,))]
    return out


def n_params():
    return int(sum(np.prod(s) for _, s in layout()))


def unpack(theta):
    P, o = {}, 0
    for name, shape in layout():
        k = int(np.prod(shape))
        P[name] = np.asarray(theta[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return P


def pack(P):
    return np.concatenate([np.asarray(P[name], dtype=np.float64).ravel() for name, _ in layout()])


def bf16(x):
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    b = x32.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


class System:
    """A free-node system as full symmetric CSR (diagonal included) plus its CNT chains."""

    def __init__(self, row_ptr, col_ind, values, chain_start, chain_len):
        self.rp = np.asarray(row_ptr, np.int64)
        self.ci = np.asarray(col_ind, np.int64)
        self.v = np.asarray(values, np.float64)
        self.n = len(self.rp) - 1
        n = self.n
        self.row = np.repeat(np.arange(n), np.diff(self.rp))
        self.diag = np.zeros(n)
        dm = self.ci == self.row
        self.diag[self.row[dm]] = self.v[dm]
        chain = np.full(n, -1, np.int64)
        pos = np.zeros(n, np.int64)
        for c, (s, l) in enumerate(zip(chain_start, chain_len)):
            chain[s:s + l] = c
            pos[s:s + l] = np.arange(l)
        self.chain = chain
        self.blk = np.cumsum((pos % BLOCK_MAX == 0) | np.r_[True, chain[1:] != chain[:-1]]) - 1
        off = ~dm
        self.off = off
        same_chain = (chain[self.row] == chain[self.ci]) & (np.abs(self.row - self.ci) == 1)
        self.jf = (off & ~same_chain).astype(np.float64)
        self.offblock = off & (self.blk[self.row] != self.blk[self.ci])
        self.deg = np.bincount(self.row[off], minlength=n).astype(np.float64)
        ld = np.log(self.diag)
        absv = np.abs(self.v)
        with np.errstate(divide="ignore"):
            la = np.where(off & (absv > 0), np.log(np.where(absv > 0, absv, 1.0)), 0.0)
        self.lc = np.where(off, la - 0.5 * (ld[self.row] + ld[self.ci]), 0.0)
        mu, sd = ld.mean(), ld.std()
        self.f = np.stack([(ld - mu) / (sd if sd > 0 else 1.0), np.log1p(self.deg)], 1)
        self._blocks()

    def _blocks(self):
        """Tridiagonal blocks: (start, m, diag d, upper e, singular flag)."""
        n, self.blocks = self.n, []
        starts = np.flatnonzero(np.r_[True, self.blk[1:] != self.blk[:-1]])
        ends = np.r_[starts[1:], n]
        up = {}
        for k in np.flatnonzero(self.off & (self.ci == self.row + 1)):
            up[int(self.row[k])] = self.v[k]
        for s, e in zip(starts, ends):
            m = e - s
            d = self.diag[s:e].copy()
            u = np.array([up.get(int(i), 0.0) if i + 1 < e else 0.0 for i in range(s, e)])
            piv = np.empty(m)
            piv[0] = d[0]
            sing = not (piv[0] > 1e-13 * abs(d[0]))
            for k in range(1, m):
                piv[k] = d[k] - (u[k - 1] / piv[k - 1]) * u[k - 1]
                sing |= not (piv[k] > 1e-13 * abs(d[k]))
            self.blocks.append((s, m, d, u, sing))

    def matvec(self, x):
        out = np.zeros(self.n)
        np.add.at(out, self.row, self.v * x[self.ci])
        return out

    def tsolve(self, r):
        z = np.empty(self.n)
        for s, m, d, u, sing in self.blocks:
            if sing:
                z[s:s + m] = r[s:s + m] / d
                continue
            T = np.diag(d) + np.diag(u[:-1], 1) + np.diag(u[:-1], -1)
            z[s:s + m] = np.linalg.solve(T, r[s:s + m])
        return z


def forward(theta, S: System, rounding=True):
    rnd = bf16 if rounding else (lambda x: np.asarray(x, np.float64))
    P = unpack(theta)
    c = {"H": [], "A": [], "G": [], "gate": []}
    A0 = S.f @ rnd(P["W_in"]) + P["b_in"]
    H = rnd(np.maximum(A0, 0))
    c["A0"] = A0
    c["H"].append(H)
    off = S.off
    rows, cols = S.row[off], S.ci[off]
    invdeg = np.where(S.deg > 0, 1.0 / np.maximum(S.deg, 1), 0.0)
    for l in range(LAYERS):
        G = rnd(H @ rnd(P[f"U{l}"]))
        p = P[f"p{l}"]
        gate = 1 / (1 + np.exp(-(p[0] * S.lc[off] + p[1] * S.jf[off] + p[2])))
        M = np.zeros_like(H)
        np.add.at(M, rows, gate[:, None] * G[cols])
        M *= invdeg[:, None]
        A = H @ rnd(P[f"W{l}"]) + M + P[f"b{l}"]
        H = rnd(H + np.maximum(A, 0))
        c["G"].append(G)
        c["gate"].append(gate)
        c["A"].append(A)
        c["H"].append(H)
    o = np.zeros(len(S.v))
    o[off] = np.sum(P["v"] * H[rows] * H[cols], 1) + P["q"][0] * S.lc[off] + P["q"][1]
    w = np.where(off, 1 / (1 + np.exp(-o)), 0.0)
    c["o"] = o
    return w, c


def precond(S: System, w, r):
    y = S.tsolve(r)
    g = np.where(S.offblock, -S.v * w, 0.0)
    u = np.zeros(S.n)
    np.add.at(u, S.row, g * y[S.ci])
    return y + S.tsolve(u), y


def loss_and_grad(theta, S: System, probes, rounding=True):
    """Mean loss over the probe vectors and its gradient w.r.t. theta (float64)."""
    P = unpack(theta)
    w, c = forward(theta, S, rounding)
    dw = np.zeros(len(S.v))
    L = 0.0
    for u0 in probes:
        r = S.matvec(u0)
        z, y = precond(S, w, r)
        q = S.matvec(z)
        rq, rr, qq = r @ q, r @ r, q @ q
        L += 1 - rq * rq / (rr * qq)
        dq = -2 * rq / (rr * qq) * r + 2 * rq * rq / (rr * qq * qq) * q
        dz = S.matvec(dq)
        lam = S.tsolve(dz)
        dw += np.where(S.offblock, lam[S.row] * (-S.v) * y[S.ci], 0.0)
    K = len(probes)
    L /= K
    dw /= K
    # edge output
    off = S.off
    rows, cols = S.row[off], S.ci[off]
    wo = w[off]
    do = dw[off] * wo * (1 - wo)
    H = c["H"][-1]
    g = {name: np.zeros(shape) for name, shape in layout()}
    g["v"] = np.sum(do[:, None] * H[rows] * H[cols], 0)
    g["q"] = np.array([np.sum(do * S.lc[off]), np.sum(do)])
    dH = np.zeros_like(H)
    np.add.at(dH, rows, do[:, None] * P["v"] * H[cols])
    np.add.at(dH, cols, do[:, None] * P["v"] * H[rows])
    rnd = bf16 if rounding else (lambda x: np.asarray(x, np.float64))
    invdeg = np.where(S.deg > 0, 1.0 / np.maximum(S.deg, 1), 0.0)
    for l in reversed(range(LAYERS)):
        Hl, A, G, gate = c["H"][l], c["A"][l], c["G"][l], c["gate"][l]
        dA = dH * (A > 0)
        g[f"W{l}"] = Hl.T @ dA
        g[f"b{l}"] = dA.sum(0)
        dM = dA * invdeg[:, None]
        dG = np.zeros_like(G)
        np.add.at(dG, cols, gate[:, None] * dM[rows])
        dgate = np.sum(dM[rows] * G[cols], 1)
        dpre = dgate * gate * (1 - gate)
        g[f"p{l}"] = np.array([np.sum(dpre * S.lc[off]), np.sum(dpre * S.jf[off]), np.sum(dpre)])
        g[f"U{l}"] = Hl.T @ dG
        dH = dH + dA @ rnd(P[f"W{l}"]).T + dG @ rnd(P[f"U{l}"]).T
    dA0 = dH * (c["A0"] > 0)
    g["W_in"] = S.f.T @ dA0
    g["b_in"] = dA0.sum(0)
    return L, pack(g)


def init_params(seed=0):
    """Initial parameters: small random weights, edge output biased to w = 0.8."""
    rng = np.random.default_rng(seed)
    P = {}
    P["W_in"] = rng.normal(0, 0.5, (2, WIDTH))
    P["b_in"] = np.full(WIDTH, 0.1)
    for l in range(LAYERS):
        P[f"U{l}"] = rng.normal(0, 1 / np.sqrt(WIDTH), (WIDTH, WIDTH))
        P[f"W{l}"] = rng.normal(0, 0.5 / np.sqrt(WIDTH), (WIDTH, WIDTH))
        P[f"b{l}"] = np.zeros(WIDTH)
        P[f"p{l}"] = np.array([0.5, 0.0, 0.0])
    P["v"] = np.zeros(WIDTH)
    P["q"] = np.array([0.0, np.log(0.8 / 0.2)])
    return pack(P)


def chains_from_labels(lab):
    """(start, len) of the maximal runs of consecutive free nodes with one CNT id."""
    lab = np.asarray(lab)
    st = np.flatnonzero(np.r_[True, lab[1:] != lab[:-1]])
    return st, np.diff(np.r_[st, len(lab)])


def system_from_dump(z, pfx, flag):
    """System of a dumped DEA system (strict-lower SSS + diagonal) with chains from the point CNT ids."""
    rp, ci, v, dg = z[pfx + "row_ptr"], z[pfx + "col_ind"], z[pfx + "values"], z[pfx + "diag"]
    n = len(dg)
    import scipy.sparse as sp

    L = sp.csr_matrix((v, ci, rp), shape=(n, n))
    A = (L + L.T + sp.diags(dg)).tocsr()
    A.sort_indices()
    nodes, res = int(z[pfx + "nodes"][0]), int(z[pfx + "nodes"][1])
    lab = np.full(nodes, -1)
    for P, nd in zip(z[pfx + "lmm_pts"], z[pfx + "lmm_nodes"]):
        if nd >= res:
            lab[nd] = flag[P]
    st, ln = chains_from_labels(lab[res:])
    return System(A.indptr, A.indices, A.data, st, ln), A
