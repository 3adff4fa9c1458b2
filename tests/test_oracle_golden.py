"""The CPU oracle against the reference decoder's own outputs (CPU only).

Every fixture in tests/golden/ was produced by running the reference decoder
(src/pelagos/decoder.py + kernels.py, Triton-interpreted on the CPU) by
tests/golden/make_golden.py.  The oracle must reproduce each one bit for bit:
errors, found_count, iterations, the last posterior, and the selected
weights (to float32 rounding of the reference's tile-tree sum).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O


def _run(golden, **over):
    args = golden.decode_args()
    args.update(over)
    return O.decode(golden.graph, golden.syndromes, O.llr_from_priors(golden.priors),
                    gamma_legs=golden.leg_table(), **args)


def test_oracle_reproduces_reference(golden):
    out = _run(golden)
    z = golden.z
    np.testing.assert_array_equal(out["errors"], z["out_errors"])
    np.testing.assert_array_equal(out["found_count"], z["out_found_count"])
    np.testing.assert_array_equal(out["iterations"], z["out_iterations"])
    np.testing.assert_array_equal(out["valid_mask"], z["out_valid_mask"])
    unconverged = np.nonzero(out["found_count"] < golden.decode_args()["stop_nconv"])[0]
    np.testing.assert_array_equal(unconverged, z["out_unconverged_indices"])
    finite = np.isfinite(z["out_weights"])
    np.testing.assert_array_equal(np.isfinite(out["weights"]), finite)
    np.testing.assert_allclose(out["weights"][finite], z["out_weights"][finite], rtol=2e-6, atol=0)
    if "out_last_posterior" in z:
        np.testing.assert_array_equal(out["last_posterior"], z["out_last_posterior"])


def test_fixtures_discriminate_mix_rounding():
    """A fused multiply-add in the memory mix changes some fixture's posterior, so the
    fixtures would catch a kernel that rounds the mix differently from the reference."""
    from conftest import Golden

    g = Golden("bb72_resume")
    sep = _run(g, mix="separate")["last_posterior"]
    assert np.array_equal(sep, g.z["out_last_posterior"])
    for mix in ("fma_gp", "fma_lp"):
        assert not np.array_equal(_run(g, mix=mix)["last_posterior"], sep)


def test_oracle_known_answer_triangle():
    """Triangle code, error on bit 0: weight log(0.95/0.05), one iteration
    (tutorials/01_single_gpu_quickstart.ipynb:129-134; tests/test_smoke.py:75-109)."""
    from scipy.sparse import csr_matrix

    H = csr_matrix(np.array([[1, 1, 0], [0, 1, 1], [1, 0, 1]], np.uint8))
    g = O.reference_graph(H)
    syn = np.array([[1, 0, 1]], np.uint8)
    out = O.decode(g, syn, O.llr_from_priors(np.full(3, 0.05)), pre_iter=10, num_sets=2, set_max_iter=10,
                   stop_nconv=1, gamma0=0.65, gamma_legs=np.zeros((2, 3), np.float32))
    assert out["errors"].tolist() == [[1, 0, 0]]
    assert out["iterations"].tolist() == [1]
    assert abs(float(out["weights"][0]) - np.log(0.95 / 0.05)) < 1e-6


def _brute_force_ml(Hd, s, p):
    """Exact maximum-likelihood error by enumeration (tests/test_triton_against_rust.py:279-309)."""
    n = Hd.shape[1]
    wj = np.log((1 - p) / p)
    best, best_w = None, np.inf
    for x in range(1 << n):
        e = np.array([(x >> j) & 1 for j in range(n)], np.uint8)
        if np.all((Hd @ e) % 2 == s):
            w = float((e * wj).sum())
            if w < best_w - 1e-12:
                best, best_w = e, w
    return best, best_w


@pytest.mark.parametrize("n,c,seed", [(8, 4, 0), (10, 5, 1)])
def test_oracle_solutions_are_valid_and_ml_when_unique(n, c, seed):
    """Deterministic min-sum on small random codes: converged outputs satisfy the
    syndrome; where the ML solution is unique and found, the weights agree."""
    from scipy.sparse import csr_matrix

    rng = np.random.default_rng(seed)
    Hd = np.zeros((c, n), np.uint8)
    for i in range(c):
        Hd[i, rng.choice(n, size=int(rng.integers(2, min(4, n) + 1)), replace=False)] = 1
    p = rng.uniform(0.005, 0.02, size=n)
    S = np.stack([rng.integers(0, 2, size=c, dtype=np.uint8) for _ in range(8)])
    g = O.reference_graph(csr_matrix(Hd))
    out = O.decode(g, S, O.llr_from_priors(p), pre_iter=200, num_sets=1, set_max_iter=0, stop_nconv=1,
                   gamma0=0.0, gamma_legs=np.zeros((1, n), np.float32), algo="plain", alpha=1.0)
    checked = 0
    for b in range(len(S)):
        if out["found_count"][b] == 0:
            assert not np.isfinite(out["weights"][b])
            continue
        assert np.array_equal((Hd @ out["errors"][b]) % 2, S[b])
        e_ml, w_ml = _brute_force_ml(Hd, S[b], p)
        w = float((out["errors"][b] * np.log((1 - p) / p)).sum())
        assert w >= w_ml - 1e-6
        checked += 1
    assert checked > 0


def test_storage_rounding_matches_torch():
    """The oracle's binary16 / bfloat16 round-to-nearest-even equals torch's casts."""
    import torch

    rng = np.random.default_rng(0)
    x = np.concatenate([
        rng.normal(0, 10, 20000), rng.normal(0, 1e-5, 2000), rng.uniform(-70000, 70000, 2000),
        np.array([0.0, -0.0, 65504, 65519.99, 65520, 65536, 1e-8, 6e-8, 5.96e-8, np.inf, -np.inf]),
    ]).astype(np.float32)
    t = torch.from_numpy(x)
    np.testing.assert_array_equal(O.round_f16(x), t.half().float().numpy())
    np.testing.assert_array_equal(O.round_bf16(x), t.bfloat16().float().numpy())
