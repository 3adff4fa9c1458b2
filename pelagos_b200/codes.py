"""Check matrices and seeded syndrome samplers for the decoder's workloads.

Everything here is host-side numpy/scipy.  Codes:

* bivariate bicycle (BB) codes ``H_X = [A | B]`` with ``x = S_l (x) I_m``,
  ``y = I_l (x) S_m`` (``S_n`` the n x n cyclic shift), ``A = x^3 + y + y^2``,
  ``B = y^3 + x + x^2``: [[72,12,6]] for (l, m) = (6, 6) and [[144,12,12]] for
  (12, 6);
* the phenomenological space-time matrix of a BB code over ``rounds`` noisy
  syndrome rounds plus one perfect round: detector round r holds the data-error
  columns ``[A|B]`` of round r and the measurement-error columns of rounds r-1
  and r, so a measurement error of round r flips detector rounds r and r+1;
* a seeded (column weight 3, row weight 6) regular LDPC matrix built by random
  socket matching, the construction of the reference's test helper
  ``_regular_code`` (tests/test_decoder_fixes.py:73-85).

Logical failure of a decoded shot is judged with ``logical_ops`` (a basis of
``ker(H_Z) / rowspace(H_X)``, the logical operators that anticommute with a
nontrivial Z-type residual of ``H_X``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.sparse import csr_matrix


def _shift(n: int) -> np.ndarray:
    return np.roll(np.eye(n, dtype=np.uint8), 1, axis=1)


def bb_blocks(l: int, m: int) -> tuple[np.ndarray, np.ndarray]:
    """A and B of the BB code with A = x^3 + y + y^2, B = y^3 + x + x^2."""
    x = np.kron(_shift(l), np.eye(m, dtype=np.uint8))
    y = np.kron(np.eye(l, dtype=np.uint8), _shift(m))
    mp = np.linalg.matrix_power
    A = (mp(x, 3) + y + mp(y, 2)) % 2
    B = (mp(y, 3) + x + mp(x, 2)) % 2
    return A.astype(np.uint8), B.astype(np.uint8)


def bb_hx_hz(l: int, m: int) -> tuple[np.ndarray, np.ndarray]:
    A, B = bb_blocks(l, m)
    return np.hstack([A, B]), np.hstack([B.T, A.T])


def bb_code_capacity_72() -> csr_matrix:
    """[[72,12,6]] H_X (36 x 72, 216 nonzeros)."""
    return csr_matrix(bb_hx_hz(6, 6)[0])


def bb_code_capacity_144() -> csr_matrix:
    """[[144,12,12]] H_X (72 x 144, 432 nonzeros)."""
    return csr_matrix(bb_hx_hz(12, 6)[0])


def phenomenological(hx: np.ndarray, rounds: int = 12) -> csr_matrix:
    """Space-time detector matrix: (rounds+1)*C rows x rounds*(V+C) columns.

    Column block of noisy round r (0-based) = [data errors (V) | measurement errors (C)].
    """
    C, V = hx.shape
    rows = (rounds + 1) * C
    cols = rounds * (V + C)
    H = np.zeros((rows, cols), dtype=np.uint8)
    I = np.eye(C, dtype=np.uint8)
    for r in range(rounds):
        c0 = r * (V + C)
        H[r * C:(r + 1) * C, c0:c0 + V] = hx
        H[r * C:(r + 1) * C, c0 + V:c0 + V + C] = I
        H[(r + 1) * C:(r + 2) * C, c0 + V:c0 + V + C] = I
    return csr_matrix(H)


def bb_phenomenological_144(rounds: int = 12) -> csr_matrix:
    """[[144,12,12]] phenomenological matrix: 936 x 2592, 6912 nonzeros for 12 rounds."""
    return phenomenological(bb_hx_hz(12, 6)[0], rounds)


def regular_ldpc(C: int = 300, V: int = 600, seed: int = 3,
                 col_weight: int = 3, row_weight: int = 6) -> csr_matrix:
    """Seeded regular LDPC matrix by socket matching (reject repeated checks in a column)."""
    assert C * row_weight == V * col_weight
    rng = np.random.default_rng(seed)
    while True:
        sockets = np.repeat(np.arange(C), row_weight)
        rng.shuffle(sockets)
        rows = sockets.reshape(V, col_weight)
        if all(len(set(r)) == col_weight for r in rows):
            break
    return csr_matrix(
        (np.ones(col_weight * V, np.uint8),
         (rows.ravel(), np.repeat(np.arange(V), col_weight))),
        shape=(C, V),
    )


# ----------------------------------------------------------------------------- GF(2)

def gf2_rank(M: np.ndarray) -> int:
    M = (np.array(M, dtype=np.uint8) & 1).copy()
    r = 0
    rows, cols = M.shape
    for c in range(cols):
        piv = np.nonzero(M[r:, c])[0]
        if piv.size == 0:
            continue
        p = r + piv[0]
        if p != r:
            M[[r, p]] = M[[p, r]]
        nz = np.nonzero(M[:, c])[0]
        nz = nz[nz != r]
        M[nz] ^= M[r]
        r += 1
        if r == rows:
            break
    return r


def gf2_nullspace(M: np.ndarray) -> np.ndarray:
    """Basis (rows) of {x : M x = 0 mod 2}."""
    M = (np.array(M, dtype=np.uint8) & 1).copy()
    rows, cols = M.shape
    pivots = []
    r = 0
    for c in range(cols):
        if r == rows:
            break
        piv = np.nonzero(M[r:, c])[0]
        if piv.size == 0:
            continue
        p = r + piv[0]
        if p != r:
            M[[r, p]] = M[[p, r]]
        nz = np.nonzero(M[:, c])[0]
        nz = nz[nz != r]
        M[nz] ^= M[r]
        pivots.append(c)
        r += 1
    free = [c for c in range(cols) if c not in set(pivots)]
    basis = np.zeros((len(free), cols), dtype=np.uint8)
    for i, f in enumerate(free):
        basis[i, f] = 1
        for j, pc in enumerate(pivots):
            basis[i, pc] = M[j, f]
    return basis


def logical_ops(hx: np.ndarray, hz: np.ndarray) -> np.ndarray:
    """Basis of ker(H_Z) modulo rowspace(H_X): k rows; L r != 0 flags a logical error."""
    ker = gf2_nullspace(hz)
    base = np.array(hx, dtype=np.uint8) & 1
    rank = gf2_rank(base)
    out = []
    cur = base
    for v in ker:
        cand = np.vstack([cur, v[None, :]])
        rk = gf2_rank(cand)
        if rk > rank:
            out.append(v)
            cur, rank = cand, rk
    return np.array(out, dtype=np.uint8)


# ----------------------------------------------------------------------------- workloads

@dataclass
class Workload:
    """A decoding workload: matrix, priors and a way to judge logical failure."""

    name: str
    H: csr_matrix
    priors: np.ndarray
    p: float
    logicals: np.ndarray          # [k, n_data] over the data columns
    data_cols: np.ndarray         # [rounds, n_data] column indices of data errors per round

    def sample(self, shots: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
        """Seeded i.i.d. Bernoulli(priors) errors and their syndromes s = H e mod 2."""
        rng = np.random.default_rng(seed)
        err = (rng.random((shots, self.H.shape[1])) < self.priors[None, :]).astype(np.uint8)
        syn = (np.asarray((self.H @ err.T.astype(np.int64))) % 2).T.astype(np.uint8)
        return err, np.ascontiguousarray(syn)

    def logical_failures(self, err: np.ndarray, est: np.ndarray, converged: np.ndarray) -> np.ndarray:
        """True where the shot failed: unconverged, or L (e + e_hat) != 0 on the data residual."""
        res = (err ^ est)[:, self.data_cols]                  # [B, rounds, n_data]
        net = np.bitwise_xor.reduce(res, axis=1)              # accumulated data residual
        flip = (net.astype(np.int64) @ self.logicals.T.astype(np.int64)) % 2
        return (~converged.astype(bool)) | flip.any(axis=1)


def workload(name: str, p: float | None = None, rounds: int = 12) -> Workload:
    """Named workloads: bb72_cc, bb144_cc, bb144_phen, ldpc2000 (p defaults per name)."""
    if name in ("bb72_cc", "bb144_cc"):
        l, m = (6, 6) if name == "bb72_cc" else (12, 6)
        hx, hz = bb_hx_hz(l, m)
        p = {"bb72_cc": 0.05, "bb144_cc": 0.03}[name] if p is None else p
        n = hx.shape[1]
        return Workload(name, csr_matrix(hx), np.full(n, p), p, logical_ops(hx, hz),
                        np.arange(n)[None, :])
    if name == "bb144_phen":
        hx, hz = bb_hx_hz(12, 6)
        p = 0.003 if p is None else p
        H = phenomenological(hx, rounds)
        C, V = hx.shape
        cols = np.stack([r * (V + C) + np.arange(V) for r in range(rounds)])
        return Workload(name, H, np.full(H.shape[1], p), p, logical_ops(hx, hz), cols)
    if name == "ldpc2000":
        H = regular_ldpc(C=2000, V=4000, seed=3)
        p = 0.02 if p is None else p
        # A classical LDPC code has no logical operator set here: every converged shot
        # whose estimate differs from the drawn error in a codeword counts as a failure.
        V = H.shape[1]
        return Workload(name, H, np.full(V, p), p, np.zeros((0, V), np.uint8),
                        np.arange(V)[None, :])
    raise ValueError(f"unknown workload {name!r}")
