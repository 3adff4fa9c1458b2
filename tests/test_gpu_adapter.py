"""relay_bp-style adapter on the B200 (RelayDecoder, ObservableDecoderRunner) and
the GF(2) product kernel that forms syndromes and observables on the device."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from scipy.sparse import csr_matrix, random as sprandom

from pelagos_b200 import ObservableDecoderRunner, RelayBPDecoder, RelayDecoder, codes
from pelagos_b200.adapter import _DeviceCSR
from pelagos_b200.proposal import LearnedRelayBPDecoder, ProposalNet, default_weights_path, load_params

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _relay_configs(priors, **relay):
    r = {"pre_iter": 80, "num_sets": 100, "set_max_iter": 60, "stop_nconv": 5, "seed": 1234}
    r.update(relay)
    return dict(msl_config={"error_priors": priors, "gamma0": 0.65},
                relay_config=r, backend_config={"device": [0], "data_type": "float32"})


def _observables(w) -> np.ndarray:
    """Logical operators on the accumulated data errors, as a [k, V] matrix over every column."""
    O = np.zeros((w.logicals.shape[0], w.H.shape[1]), np.uint8)
    for cols in w.data_cols:
        O[:, cols] = w.logicals
    return O


def test_gf2_matvec_matches_numpy():
    rng = np.random.default_rng(3)
    A = (sprandom(50, 700, density=0.02, random_state=4, format="csr") != 0).astype(np.uint8)
    A = A.tolil()
    A[7, :] = 0  # an empty row
    A = csr_matrix(A)
    x = rng.integers(0, 2, (333, 700)).astype(np.uint8)
    got = _DeviceCSR(A, torch.device(DEV)).apply(torch.from_numpy(x).to(DEV)).cpu().numpy()
    np.testing.assert_array_equal(got, (A @ x.T.astype(np.int64) % 2).T)
    assert (got[:, 7] == 0).all()


def test_relay_decoder_matches_the_decoder():
    w = codes.workload("bb72_cc", p=0.05)
    err, syn = w.sample(512, seed=8)
    ad = RelayDecoder(w.H, **_relay_configs(w.priors))
    ref = RelayBPDecoder(w.H, w.priors, pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, stop_nconv=5,
                         seed=1234, algo="relay").decode(torch.from_numpy(syn))
    errors, iters = ad.decode_batch(syn, return_iterations=True)
    np.testing.assert_array_equal(errors, ref["errors"].cpu().numpy())
    np.testing.assert_array_equal(iters, ref["iterations"].cpu().numpy())
    one = ad.decode(syn[3])
    np.testing.assert_array_equal(one["bits"].cpu().numpy(), errors[3])
    assert one["converged"] == bool(ref["found_count"][3] > 0)
    det = ad.decode_detailed(syn[3])
    assert det.success == one["converged"] and det.iterations == int(iters[3])
    recs = ad.decode_detailed_batch_from_syndromes(syn)
    wj = ad.log_prior_ratios()
    for i in (0, 5, 100):
        assert recs[i].found_count == int(ref["found_count"][i])
        if recs[i].success:
            assert recs[i].decoding_quality == pytest.approx(float(errors[i].astype(np.float64) @ wj))


def test_valid_mask_and_found_count_through_the_adapter():
    """valid_mask == found_count >= stop_nconv; both detailed-batch methods report found_count
    (the reference's test_decoder_fixes.py:117-130 and test_unconverged_correction.py:234-248)."""
    w = codes.workload("bb72_cc", p=0.08)
    syn = w.sample(256, seed=2)[1]
    for S in (1, 2, 4):
        ad = RelayDecoder(w.H, **_relay_configs(w.priors, stop_nconv=S, pre_iter=20, num_sets=20,
                                                set_max_iter=20, seed=7))
        out = ad._decode_inner(torch.from_numpy(syn))
        found = out["found_count"].cpu()
        assert torch.equal(out["valid_mask"].cpu(), found >= S)
        for method in (ad.decode_detailed_batch, ad.decode_detailed_batch_from_syndromes):
            np.testing.assert_array_equal([r.found_count for r in method(syn)], found.numpy())


@pytest.mark.parametrize("key,value,attr", [("gamma_draw", "per_row", "gamma_draw"),
                                            ("unconverged_correction", "last_leg", "unconverged_correction")])
def test_adapter_passes_relay_options(key, value, attr):
    w = codes.workload("bb72_cc")
    ad = RelayDecoder(w.H, **_relay_configs(w.priors, **{key: value}))
    assert getattr(ad._dec, attr) == value


@pytest.mark.parametrize("learned", [False, True])
def test_observable_runner(learned):
    w = codes.workload("bb144_phen", p=0.004)
    err, syn = w.sample(4096, seed=61)
    cfg = _relay_configs(w.priors)
    if learned:
        cfg["backend_config"]["proposal"] = "default"
    ad = RelayDecoder(w.H, **cfg)
    O = _observables(w)
    runner = ObservableDecoderRunner(ad, O)
    recs = runner.from_errors_decode_observables_detailed_batch(err)
    # host restatement of the same records
    if learned:
        dec = RelayBPDecoder(w.H, w.priors, pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65,
                             stop_nconv=5, seed=1234, algo="relay")
        ref = LearnedRelayBPDecoder(dec, ProposalNet(dec, load_params(default_weights_path())[0]), gate=True)
        out = {k: v.cpu().numpy() for k, v in ref.decode(torch.from_numpy(syn)).items()}
    else:
        out = {k: v.cpu().numpy() for k, v in ad._dec.decode(torch.from_numpy(syn)).items()}
    pred = (O.astype(np.int64) @ out["errors"].T.astype(np.int64) % 2).T
    true = (O.astype(np.int64) @ err.T.astype(np.int64) % 2).T
    fails = w.logical_failures(err, out["errors"], out["found_count"] > 0)
    wj = ad.log_prior_ratios()
    for i, r in enumerate(recs):
        np.testing.assert_array_equal(r.decoding, out["errors"][i])
        np.testing.assert_array_equal(r.observables, pred[i])
        assert r.iterations == out["iterations"][i]
        assert r.error_detected == bool((pred[i] != true[i]).any())
        assert r.success == bool(out["found_count"][i] > 0)
        assert (r.error_detected or not r.success) == bool(fails[i])
        if r.success:
            assert r.decoding_quality == pytest.approx(float(out["errors"][i].astype(np.float64) @ wj))
