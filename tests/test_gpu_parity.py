"""CUDA decoder parity (B200).

* every reference fixture, decoded through RelayBPDecoder (the C ABI + sm_100a
  kernel), reproduces the reference's outputs bit for bit;
* seeded [[72,12,6]] and [[144,12,12]]-phenomenological batches match the CPU
  oracle bit for bit in every message precision;
* full-size properties: every converged shot reproduces its syndrome, and
  results do not depend on batch composition, order or launch shape.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import oracle as O
from pelagos_b200 import RelayBPDecoder, codes

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)
KEYS = ("errors", "found_count", "iterations", "weight_fixed")


def _np(out):
    return {k: v.cpu().numpy() for k, v in out.items() if isinstance(v, torch.Tensor)}


def _golden_decoder(g, **extra):
    kw = {k: (tuple(v) if isinstance(v, list) else v) for k, v in g.kw.items()}
    R = g.num_sets
    if R > 0:
        legs = g.leg_table()
        kw["explicit_gammas"] = np.stack([legs[(j - 1) % R] for j in range(R)])
        kw.pop("gamma_dist_interval_by_error", None)
    kw.pop("kw_explicit_gammas", None)
    kw.update(extra)
    return RelayBPDecoder(g.H, g.priors, **kw)


def _golden_decode_kwargs(g):
    d = {}
    for k in ("init_posterior", "init_gamma", "prior_llr"):
        if f"dkw_{k}" in g.z:
            d[k] = torch.from_numpy(g.z[f"dkw_{k}"]).to(DEV)
    for k in ("pre_iter_override", "skip_relay_legs", "return_last_posterior"):
        if k in g.dkw:
            d[k] = g.dkw[k]
    return d


#: kernel families, as (groups_per_block, shots_per_group): the block-per-group kernel with one
#: and with two shots per group, and the (default) kernel whose blocks hold several one-shot groups
NSHOTS = [(1, 1), (1, 2), (0, 1), (1, 1, 2)]  # block-per-group (one, two shots), multi-group, two blocks per SM


@pytest.mark.parametrize("nshots", NSHOTS)
def test_reference_fixtures_bit_exact(golden, nshots):
    try:
        dec = _golden_decoder(golden, launch=(0, *nshots))
    except NotImplementedError:
        if nshots == (0, 1):
            raise
        pytest.skip("the block-per-group kernel covers check degrees up to 16")
    out = _np(dec.decode(torch.from_numpy(golden.syndromes).to(DEV), **_golden_decode_kwargs(golden)))
    z = golden.z
    np.testing.assert_array_equal(out["errors"], z["out_errors"])
    np.testing.assert_array_equal(out["found_count"], z["out_found_count"])
    np.testing.assert_array_equal(out["iterations"], z["out_iterations"])
    np.testing.assert_array_equal(out["valid_mask"], z["out_valid_mask"])
    np.testing.assert_array_equal(out["unconverged_indices"], z["out_unconverged_indices"])
    fin = np.isfinite(z["out_weights"])
    np.testing.assert_array_equal(np.isfinite(out["weights"]), fin)
    np.testing.assert_allclose(out["weights"][fin], z["out_weights"][fin], rtol=2e-6)
    if "out_last_posterior" in z:
        np.testing.assert_array_equal(out["last_posterior"].astype(np.float64), z["out_last_posterior"])


def _oracle_for(dec: RelayBPDecoder, syn, data_type=None, **kw):
    g = O.reference_graph(dec.H_csr)
    return O.decode(g, syn, dec.log_prior_ratios, pre_iter=kw.pop("pre_iter", dec.pre_iter),
                    num_sets=dec.num_sets, set_max_iter=dec.set_max_iter, stop_nconv=dec.stop_nconv,
                    gamma0=dec.gamma0, gamma_legs=dec._leg_table(0), algo=dec.algo,
                    last_leg=dec.unconverged_correction == "last_leg", alpha=dec.normalized_min_sum_alpha,
                    alpha_scaling=dec.alpha_iteration_scaling_factor, beta=dec.offset_min_sum_beta,
                    data_type=data_type or dec.dtype_str, **kw)


def _assert_same(out, ref, keys=KEYS):
    for k in keys:
        a, b = out[k], ref[k]
        if not np.array_equal(a, b):
            bad = np.nonzero((a != b).reshape(len(a), -1).any(1))[0]
            raise AssertionError(f"{k} differs on {len(bad)} shots, first {bad[:8].tolist()}")


@pytest.mark.parametrize("nshots", NSHOTS)
@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16", "float64"])
def test_bb72_code_capacity_matches_oracle(dtype, nshots):
    w = codes.workload("bb72_cc")
    err, syn = w.sample(1024 if dtype == "float32" else 256, seed=7)
    dec = RelayBPDecoder(w.H, w.priors, data_type=dtype, launch=(0, *nshots), **RELAY)
    out = _np(dec.decode(torch.from_numpy(syn).to(DEV), return_last_posterior=True))
    ref = _oracle_for(dec, syn)
    _assert_same(out, ref)
    np.testing.assert_array_equal(out["last_posterior"].astype(np.float64), ref["last_posterior"])


@pytest.mark.parametrize("nshots", NSHOTS)
@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_bb144_phenomenological_matches_oracle(dtype, nshots):
    w = codes.workload("bb144_phen")
    err, syn = w.sample(384, seed=11)
    dec = RelayBPDecoder(w.H, w.priors, data_type=dtype, launch=(0, *nshots), **RELAY)
    out = _np(dec.decode(torch.from_numpy(syn).to(DEV)))
    _assert_same(out, _oracle_for(dec, syn))


@pytest.mark.parametrize("variant", [
    dict(stop_nconv=1), dict(stop_nconv=2, pre_iter=0), dict(num_sets=0), dict(algo="plain"),
    dict(normalized_min_sum_alpha=0.0, alpha_iteration_scaling_factor=2.0), dict(offset_min_sum_beta=0.3),
    dict(unconverged_correction="last_leg"), dict(set_max_iter=0), dict(pre_iter=3, num_sets=5, set_max_iter=4),
    dict(mix_rounding="fma_gp"), dict(mix_rounding="fma_lp"),
])
@pytest.mark.parametrize("nshots", NSHOTS)
def test_options_match_oracle(variant, nshots):
    w = codes.workload("bb72_cc", p=0.08)
    err, syn = w.sample(512, seed=3)
    variant = dict(variant)
    kw = dict(RELAY)
    kw.update(pre_iter=20, num_sets=12, set_max_iter=15)
    mix = variant.pop("mix_rounding", "separate")
    kw.update(variant)
    dec = RelayBPDecoder(w.H, w.priors, mix_rounding=mix, launch=(0, *nshots), **kw)
    out = _np(dec.decode(torch.from_numpy(syn).to(DEV)))
    _assert_same(out, _oracle_for(dec, syn, mix=mix))


@pytest.mark.parametrize("nshots", NSHOTS)
def test_per_shot_inputs_match_oracle(nshots):
    w = codes.workload("bb144_cc")
    err, syn = w.sample(256, seed=5)
    rng = np.random.default_rng(9)
    V = w.H.shape[1]
    ip = (3.4 + rng.normal(0, 1.5, (256, V))).astype(np.float32)
    ig = rng.uniform(-0.2, 0.8, (256, V)).astype(np.float32)
    pl = rng.uniform(2.5, 4.5, (256, V)).astype(np.float32)
    lg = rng.uniform(-0.24, 0.66, (256, 3, V)).astype(np.float32)
    kw = dict(RELAY, pre_iter=25, num_sets=8, set_max_iter=20, stop_nconv=3)
    dec = RelayBPDecoder(w.H, w.priors, launch=(0, *nshots), **kw)
    t = lambda a: torch.from_numpy(a).to(DEV)  # noqa: E731
    out = _np(dec.decode(t(syn), init_posterior=t(ip), init_gamma=t(ig), prior_llr=t(pl), leg_gammas=t(lg),
                         pre_iter_override=30, return_last_posterior=True))
    ref = _oracle_for(dec, syn, pre_iter=30, init_posterior=ip, gamma_pre=ig, llr_per_shot=pl,
                      gamma_legs_shot=lg)
    _assert_same(out, ref)
    np.testing.assert_array_equal(out["last_posterior"].astype(np.float64), ref["last_posterior"])


def test_per_row_gamma_draw_matches_oracle():
    w = codes.workload("bb72_cc", p=0.08)
    err, syn = w.sample(128, seed=4)
    dec = RelayBPDecoder(w.H, w.priors, gamma_draw="per_row", **dict(RELAY, num_sets=6, stop_nconv=3))
    out = _np(dec.decode(torch.from_numpy(syn).to(DEV)))
    legs = dec._per_row_legs(128, 0, 0).cpu().numpy()
    _assert_same(out, _oracle_for(dec, syn, gamma_legs_shot=legs))


def test_bitpack_output():
    from pelagos_b200.utils import bitunpack_errors

    w = codes.workload("bb72_cc")
    err, syn = w.sample(300, seed=8)
    s = torch.from_numpy(syn).to(DEV)
    a = RelayBPDecoder(w.H, w.priors, **RELAY).decode(s)
    b = RelayBPDecoder(w.H, w.priors, bitpack_output=True, **RELAY).decode(s)
    assert b["errors"].dtype == torch.int32 and b["errors"].shape == (300, 3)
    assert torch.equal(bitunpack_errors(b["errors"].cpu(), 72), a["errors"].cpu())


def test_empty_and_single_batches():
    w = codes.workload("bb72_cc")
    err, syn = w.sample(5, seed=1)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    out = dec.decode(torch.zeros(0, 36, dtype=torch.uint8, device=DEV))
    assert out["errors"].shape == (0, 72) and out["unconverged_indices"].numel() == 0
    full = _np(dec.decode(torch.from_numpy(syn).to(DEV)))
    for i in range(5):
        one = _np(dec.decode(torch.from_numpy(syn[i:i + 1])))  # host tensor input
        for k in KEYS:
            np.testing.assert_array_equal(one[k][0], full[k][i])


def test_bad_shapes_raise():
    w = codes.workload("bb72_cc")
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    with pytest.raises(ValueError, match="syndrome bits"):
        dec.decode(torch.zeros(2, 35, dtype=torch.uint8, device=DEV))
    with pytest.raises(ValueError, match="init_posterior"):
        dec.decode(torch.zeros(2, 36, dtype=torch.uint8, device=DEV),
                   init_posterior=torch.zeros(3, 72, device=DEV))


def test_constructor_errors_mirror_reference():
    w = codes.workload("bb72_cc")
    with pytest.raises(ValueError, match="Unknown algo"):
        RelayBPDecoder(w.H, w.priors)
    with pytest.raises(ValueError, match="gamma_draw"):
        RelayBPDecoder(w.H, w.priors, algo="relay", gamma_draw="shared")
    with pytest.raises(ValueError, match="first_leg.*last_leg"):
        RelayBPDecoder(w.H, w.priors, algo="relay", unconverged_correction="x")
    with pytest.raises(ValueError, match="data_type"):
        RelayBPDecoder(w.H, w.priors, algo="relay", data_type="int8")


@pytest.fixture(scope="module")
def bb144_full():
    w = codes.workload("bb144_phen")
    err, syn = w.sample(65536, seed=2026)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    out = _np(dec.decode(torch.from_numpy(syn).to(DEV)))
    return w, err, syn, dec, out


def test_full_size_syndrome_consistency(bb144_full):
    """[[144,12,12]] phenomenological, 65,536 shots: every converged shot's errors satisfy H e = s."""
    w, err, syn, dec, out = bb144_full
    solved = out["found_count"] > 0
    assert solved.mean() > 0.99
    e = out["errors"][solved].astype(np.int64)
    res = (w.H @ e.T) % 2
    np.testing.assert_array_equal(res.T.astype(np.uint8), syn[solved])
    assert np.all(np.isfinite(out["weights"][solved])) and not np.any(np.isfinite(out["weights"][~solved]))
    np.testing.assert_array_equal(out["valid_mask"], out["found_count"] >= 5)


def test_full_size_batch_and_permutation_invariance(bb144_full):
    w, err, syn, dec, out = bb144_full
    rng = np.random.default_rng(1)
    idx = rng.permutation(len(syn))[:4096]
    sub = _np(dec.decode(torch.from_numpy(syn[idx]).to(DEV)))
    for k in KEYS:
        np.testing.assert_array_equal(sub[k], out[k][idx])


@pytest.mark.parametrize("shape", [(192, 1), (256, 1), (448, 1), (512, 1), (768, 1), (864, 1),
                                   (256, 1, 2), (384, 1, 2), (448, 1, 2), (480, 1, 2),
                                   (256, 1, 1, 2), (352, 1, 1, 2), (384, 1, 1, 2), (448, 1, 1, 2)])
def test_launch_shape_invariance(shape):
    w = codes.workload("bb144_phen")
    err, syn = w.sample(512, seed=12)
    a = RelayBPDecoder(w.H, w.priors, **RELAY)
    b = RelayBPDecoder(w.H, w.priors, launch=shape, **RELAY)
    s = torch.from_numpy(syn).to(DEV)
    oa, ob = _np(a.decode(s)), _np(b.decode(s))
    for k in KEYS:
        np.testing.assert_array_equal(oa[k], ob[k])


@pytest.mark.parametrize("pre,legs", [((352, 1, 1, 2), (704, 1, 1)), ((704, 1, 1), (352, 1, 1, 2)),
                                      ((448, 1, 1, 2), (384, 1, 1, 2))])
def test_per_kind_launch_shapes(pre, legs):
    """The pre-iteration launch and the relay-leg launch of a two-launch decode take their own
    shapes (reported by launch_info) and give the single-shape result."""
    w = codes.workload("bb144_phen")
    err, syn = w.sample(2048, seed=21)
    a = RelayBPDecoder(w.H, w.priors, **RELAY)
    b = RelayBPDecoder(w.H, w.priors, **RELAY)
    b.configure_launch(*legs, kind="legs")
    b.configure_launch(*pre, kind="pre")
    info = b.launch_info()
    assert (info["group_threads"], info["blocks_per_sm"]) == (legs[0], legs[3] if len(legs) > 3 else 1)
    assert (info["pre"]["group_threads"], info["pre"]["blocks_per_sm"]) == (pre[0], pre[3] if len(pre) > 3 else 1)
    for shape, i in ((pre, info["pre"]), (legs, info)):
        assert i["blocks"] == (2 if len(shape) > 3 else 1) * torch.cuda.get_device_properties(0).multi_processor_count
    s = torch.from_numpy(syn).to(DEV)
    oa, ob = _np(a.decode(s)), _np(b.decode(s))
    for k in KEYS:
        np.testing.assert_array_equal(oa[k], ob[k])


def test_two_blocks_per_sm_rejects_shapes_outside_its_budget():
    w = codes.workload("bb144_phen")
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    with pytest.raises(NotImplementedError, match="register budget"):
        dec.configure_launch(704, 1, 1, 2)     # 4 variables per thread: at most 512 threads
    with pytest.raises(NotImplementedError, match="register budget"):
        dec.configure_launch(480, 1, 1, 2)     # 6 variables per thread: at most 448 threads
    with pytest.raises(NotImplementedError, match="two blocks per SM"):
        dec.configure_launch(352, 1, 2, 2)     # two-shot groups keep one block per SM
    with pytest.raises(ValueError, match="blocks_per_sm"):
        dec.configure_launch(352, 1, 1, 3)
