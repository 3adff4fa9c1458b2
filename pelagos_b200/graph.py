"""Tanner graph of a check matrix in the reference's edge-centric form.

Mirrors ``CSRGraph._build_edge_representation`` (src/pelagos/graph.py:101-211):

* edge ``e`` is the e-th stored entry of the CSR matrix (row by row, in the
  matrix's own column order, sorted or not);
* ``chk_ptr`` = CSR ``indptr``; ``edge_var[e]`` = column of edge e;
* ``var_edges`` = ``np.argsort(edge_var)`` with numpy's default (non-stable)
  sort, the exact call of graph.py:145, so each variable sums its incoming
  messages in the same order as the reference on the same machine;
  ``var_ptr`` delimits each variable's block.

The device layout the kernel uses (check-slot-major message slots and the
per-variable slot table) is derived from these arrays inside the native
library (rbp_graph_create).
"""

from __future__ import annotations

import hashlib

import numpy as np
from scipy.sparse import csr_matrix, issparse


class TannerGraph:
    """Host arrays of the edge-centric graph (int32)."""

    def __init__(self, H_csr, check_permutation=None):
        if not issparse(H_csr):
            raise ValueError("Input must be a scipy.sparse matrix")
        if not isinstance(H_csr, csr_matrix):
            H_csr = H_csr.tocsr()
        self.C, self.V = H_csr.shape
        if H_csr.dtype != np.uint8 and H_csr.dtype != bool:
            H_csr = (H_csr != 0).astype(np.uint8)
        if check_permutation is not None:
            perm = np.asarray(check_permutation, dtype=np.int32)
            if perm.shape[0] != H_csr.shape[0]:
                raise ValueError(
                    f"check_permutation length ({perm.shape[0]}) must match number of checks ({H_csr.shape[0]})")
            if not (perm.min() >= 0 and perm.max() < H_csr.shape[0]):
                raise ValueError(f"check_permutation indices must be in range [0, {H_csr.shape[0]})")
            H_csr = H_csr[perm, :]
        self.H = H_csr
        self.E = int(H_csr.nnz)
        self.chk_ptr = H_csr.indptr.astype(np.int32)
        self.edge_var = H_csr.indices.astype(np.int32)
        self.edge_chk = np.repeat(np.arange(self.C, dtype=np.int32), np.diff(self.chk_ptr))
        self.var_edges = np.argsort(self.edge_var).astype(np.int32)
        counts = np.bincount(self.edge_var, minlength=self.V)
        self.var_ptr = np.zeros(self.V + 1, dtype=np.int32)
        np.cumsum(counts, out=self.var_ptr[1:])
        self.max_deg_chk = int(np.diff(self.chk_ptr).max()) if self.C else 0
        self.max_deg_var = int(counts.max()) if self.V else 0

    @property
    def sparsity_hash(self) -> str:
        """Hash of the degree distributions and per-check sorted column sets (cf. graph.py:183-211)."""
        cd = np.sort(np.diff(self.chk_ptr)).astype(np.int32)
        vd = np.sort(np.diff(self.var_ptr)).astype(np.int32)
        rows = [np.sort(self.edge_var[self.chk_ptr[c]:self.chk_ptr[c + 1]]) for c in range(self.C)]
        blob = np.concatenate([cd, vd, np.concatenate(rows).astype(np.int32)]).tobytes()
        return hashlib.blake2b(blob, digest_size=16).hexdigest()

    def get_stats(self) -> dict:
        return {
            "checks": self.C,
            "variables": self.V,
            "edges": self.E,
            "max_degree_check": self.max_deg_chk,
            "max_degree_variable": self.max_deg_var,
            "avg_degree_check": self.E / self.C,
            "avg_degree_variable": self.E / self.V,
        }

    def validate(self) -> bool:
        assert self.edge_var.max() < self.V and self.edge_chk.max() < self.C
        assert self.chk_ptr.shape[0] == self.C + 1 and self.var_ptr.shape[0] == self.V + 1
        assert np.all(np.diff(self.chk_ptr) >= 0) and np.all(np.diff(self.var_ptr) >= 0)
        assert self.chk_ptr[-1] == self.E and self.var_ptr[-1] == self.E
        assert np.array_equal(self.edge_var[self.var_edges], np.repeat(np.arange(self.V), np.diff(self.var_ptr)))
        return True
