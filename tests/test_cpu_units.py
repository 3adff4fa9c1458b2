"""Host-side units (CPU only): priors, validation, bit packing, gamma draws, graph, codes.

Mirrors the reference's tests/test_cpu_units.py and tests/test_gamma_sampling.py
for the functions this package re-implements with the same names.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from scipy.sparse import csc_matrix, csr_matrix

from pelagos_b200 import codes
from pelagos_b200.graph import TannerGraph
from pelagos_b200.utils import (
    alpha_schedule,
    bitpack_errors,
    bitunpack_errors,
    compute_log_prior_ratios,
    sample_gamma_per_variable,
    sample_gamma_uniform,
    validate_csr_matrix,
    validate_error_priors,
)


def test_log_prior_ratios_match_formula():
    p = np.array([0.001, 0.01, 0.1, 0.3])
    llr = compute_log_prior_ratios(p)
    assert llr.dtype == np.float32
    np.testing.assert_allclose(llr, np.log((1 - p) / p), rtol=1e-6)


def test_log_prior_ratios_are_finite_for_zero_prior():
    llr = compute_log_prior_ratios(np.array([0.0, 0.05]))
    assert np.all(np.isfinite(llr)) and llr[0] > llr[1]


def test_validate_error_priors(capsys):
    p = np.array([0.001, 0.2, 0.45])
    np.testing.assert_array_equal(validate_error_priors(p), p)
    with pytest.raises(ValueError, match="1D"):
        validate_error_priors(np.full((2, 3), 0.01))
    validate_error_priors(np.array([0.0, 0.7]))
    assert "clipped" in capsys.readouterr().out


def test_validate_csr_matrix():
    H = np.array([[1, 1, 0], [0, 1, 1]], dtype=np.uint8)
    assert validate_csr_matrix(csr_matrix(H)) and validate_csr_matrix(csc_matrix(H))
    for bad, msg in [(np.array([[1, 0], [0, 1]]), "scipy.sparse"),
                     (csr_matrix((0, 3), dtype=np.uint8), "empty"),
                     (csr_matrix((2, 3), dtype=np.uint8), "zero non-zero")]:
        with pytest.raises(ValueError, match=msg):
            validate_csr_matrix(bad)


@pytest.mark.parametrize("V", [1, 31, 32, 33, 100])
def test_bitpack_roundtrip(V):
    rng = np.random.default_rng(V)
    errors = torch.from_numpy(rng.integers(0, 2, size=(4, V), dtype=np.uint8))
    packed = bitpack_errors(errors)
    assert packed.shape == (4, (V + 31) // 32) and packed.dtype == torch.int32
    assert torch.equal(bitunpack_errors(packed, V), errors)


def test_bitpack_word_layout():
    e = torch.zeros(1, 33, dtype=torch.uint8)
    e[0, 0] = e[0, 31] = e[0, 32] = 1
    p = bitpack_errors(e)
    assert p[0, 0].item() == (1 | -(1 << 31)) and p[0, 1].item() == 1


def test_gamma_draw_matches_manual_seed():
    """tests/test_gamma_sampling.py:49-63 on CPU: the draw equals manual_seed + rand."""
    B, V, seed = 64, 257, 1237
    got = sample_gamma_uniform(B, V, 0.1, 0.9, "cpu", seed)
    torch.manual_seed(seed)
    assert torch.equal(got, 0.1 + (0.9 - 0.1) * torch.rand(B, V))
    low = torch.arange(V, dtype=torch.float32) / V
    iv = torch.stack([low, low + 0.5], 1)
    got = sample_gamma_per_variable(B, V, iv, "cpu", seed)
    torch.manual_seed(seed)
    u = torch.rand(B, V)
    assert torch.equal(got, low[None] + ((low + 0.5)[None] - low[None]) * u)


def test_gamma_draw_leaves_global_rng_alone():
    torch.manual_seed(999)
    before = torch.random.get_rng_state()
    sample_gamma_uniform(4, 9, -0.24, 0.66, "cpu", 5)
    assert torch.equal(torch.random.get_rng_state(), before)


def test_alpha_schedule():
    use, t = alpha_schedule(None, 1.0, 3)
    assert not use
    use, t = alpha_schedule(0.0, 2.0, 3)
    assert use and np.allclose(t, [1 - 2 ** -0.5, 1 - 2 ** -1.0, 1 - 2 ** -1.5]) and t.dtype == np.float32
    use, t = alpha_schedule(0.8, 1.0, 2)
    assert use and np.all(t == np.float32(0.8))


def test_graph_matches_reference_fixture_order(golden):
    """var_edges / var_ptr / edge_var equal the reference graph's arrays for every fixture."""
    g = TannerGraph(golden.H)
    assert g.validate()
    np.testing.assert_array_equal(g.edge_var, golden.z["ref_edge_var"])
    np.testing.assert_array_equal(g.var_ptr, golden.z["ref_var_ptr"])
    np.testing.assert_array_equal(g.var_edges, golden.z["ref_var_edges"])


def test_graph_unsorted_csr_keeps_row_order():
    H = csr_matrix(np.array([[1, 0, 1, 0], [0, 1, 1, 1]], np.uint8))
    Hu = csr_matrix((H.data, H.indices[::-1].copy(), H.indptr), shape=H.shape)
    g = TannerGraph(Hu)
    np.testing.assert_array_equal(g.edge_var, Hu.indices)
    assert g.validate()


@pytest.mark.parametrize("lm,k", [((6, 6), 12), ((12, 6), 12)])
def test_bb_codes(lm, k):
    hx, hz = codes.bb_hx_hz(*lm)
    assert not ((hx.astype(int) @ hz.T.astype(int)) % 2).any()
    assert hx.shape[1] - 2 * codes.gf2_rank(hx) == k
    L = codes.logical_ops(hx, hz)
    assert L.shape[0] == k
    assert not ((hz.astype(int) @ L.T.astype(int)) % 2).any()


def test_phenomenological_shape():
    H = codes.bb_phenomenological_144()
    assert H.shape == (936, 2592) and H.nnz == 6912
    assert set(np.diff(H.indptr).tolist()) == {1, 7, 8}
    assert set(np.diff(H.tocsc().indptr).tolist()) == {2, 3}


def test_regular_ldpc():
    H = codes.regular_ldpc(300, 600, 3)
    assert H.shape == (300, 600) and H.nnz == 1800
    assert set(np.diff(H.tocsc().indptr).tolist()) == {3}
    assert set(np.diff(H.indptr).tolist()) == {6}


def test_workload_sampling_and_failures():
    w = codes.workload("bb72_cc")
    err, syn = w.sample(200, seed=1)
    np.testing.assert_array_equal(syn, (err.astype(int) @ w.H.T.toarray().astype(int)) % 2)
    ok = np.ones(200, bool)
    assert not w.logical_failures(err, err, ok).any()
    assert w.logical_failures(err, err, ~ok).all()
    # adding a stabilizer (row of H_Z) is not a logical error; a logical operator is
    hx, hz = codes.bb_hx_hz(6, 6)
    assert not w.logical_failures(err[:1], err[:1] ^ hz[0], ok[:1]).any()
    ker = codes.gf2_nullspace(hx)
    flips = [w.logical_failures(err[:1], err[:1] ^ v, ok[:1])[0] for v in ker]
    assert any(flips)
