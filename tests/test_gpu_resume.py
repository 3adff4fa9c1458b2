"""Resumable decoding, the leg-synchronous early exit and the unconverged correction (B200).

A decode can stop after the pre-iterations or after any relay leg, save each
shot's state (best solution, counters, hard-decision source, posterior) and be
resumed from the next leg.  Because each shot's legs only depend on its own
state and on the fixed leg draws, any split must give bit-for-bit the outputs
of the uninterrupted decode, and a decode stopped after k legs must equal the
decoder built with ``num_sets=k``.

``fast_max_unconverged_pct`` runs that way, one leg per launch, and stops once
the unconverged fraction falls below the threshold (reference
src/pelagos/decoder.py:2890-2935, 3658-3662, 3812-3831).  The unconverged
correction cases mirror the reference's tests/test_unconverged_correction.py.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch
from scipy.sparse import csr_matrix

from pelagos_b200 import RelayBPDecoder, codes

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)
KEYS = ("errors", "found_count", "iterations", "weight_fixed", "valid_mask", "weights")


def _np(out):
    return {k: v.cpu().numpy() for k, v in out.items() if isinstance(v, torch.Tensor)}


def _same(a, b, keys=KEYS, what=""):
    for k in keys:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{what} {k}")


@pytest.fixture(scope="module")
def bb144():
    w = codes.workload("bb144_phen", p=0.004)
    syn = torch.from_numpy(w.sample(4096, seed=91)[1]).to(DEV)
    return w, syn


@pytest.mark.parametrize("dtype", ["float32", "float64", "bfloat16"])
def test_split_after_pre_iterations_matches_full(bb144, dtype):
    w, syn = bb144
    dec = RelayBPDecoder(w.H, w.priors, data_type=dtype, **RELAY)
    full = _np(dec.decode(syn, return_last_posterior=True))
    state = dec.new_state(syn.shape[0])
    dec.decode_phases(syn, suspend=state, skip_relay_legs=True)
    got = _np(dec.decode_phases(syn, resume=state, legs_begin=0, return_last_posterior=True))
    _same(got, full, KEYS + ("last_posterior",), dtype)


@pytest.mark.parametrize("k", [1, 2, 5])
def test_split_after_leg_k_matches_full_and_truncated(bb144, k):
    w, syn = bb144
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    full = _np(dec.decode(syn))
    state = dec.new_state(syn.shape[0])
    part = _np(dec.decode_phases(syn, suspend=state, legs_end=k))
    trunc = _np(RelayBPDecoder(w.H, w.priors, **{**RELAY, "num_sets": k}).decode(syn))
    _same(part, trunc, what=f"stopped after {k} legs vs num_sets={k}")
    got = _np(dec.decode_phases(syn, resume=state, legs_begin=k))
    _same(got, full, what=f"resumed at leg {k}")


def test_one_leg_per_launch_matches_full(bb144):
    w, syn = bb144
    cfg = {**RELAY, "num_sets": 12}
    dec = RelayBPDecoder(w.H, w.priors, **cfg)
    full = _np(dec.decode(syn, return_last_posterior=True))
    a, b = dec.new_state(syn.shape[0]), dec.new_state(syn.shape[0])
    dec.decode_phases(syn, suspend=a, skip_relay_legs=True)
    for leg in range(cfg["num_sets"]):
        out = dec.decode_phases(syn, resume=a, suspend=b, legs_begin=leg, legs_end=leg + 1,
                                return_last_posterior=True)
        a, b = b, a
    _same(_np(out), full, KEYS + ("last_posterior",))


def test_resume_in_place(bb144):
    """resume and suspend may name the same buffer (each shot reads its state before writing it)."""
    w, syn = bb144
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    full = _np(dec.decode(syn))
    st = dec.new_state(syn.shape[0])
    dec.decode_phases(syn, suspend=st, legs_end=3)
    dec.decode_phases(syn, resume=st, suspend=st, legs_begin=3, legs_end=7)
    _same(_np(dec.decode_phases(syn, resume=st, legs_begin=7)), full)


def test_fast_max_zero_runs_every_leg(bb144):
    w, syn = bb144
    full = _np(RelayBPDecoder(w.H, w.priors, **RELAY).decode(syn))
    got = RelayBPDecoder(w.H, w.priors, fast_max_unconverged_pct=0.0, **RELAY).decode(syn)
    _same(_np(got), full)
    np.testing.assert_array_equal(got["unconverged_indices"].cpu().numpy(),
                                  np.nonzero(full["found_count"] < RELAY["stop_nconv"])[0])


def test_fast_max_stops_at_first_leg_under_threshold(bb144):
    """The exit comes after the first phase whose unconverged fraction is below the threshold; the
    outputs are those of the decoder truncated to that many legs."""
    w, syn = bb144
    S = RELAY["stop_nconv"]
    fracs = []
    for k in range(0, 10):
        o = _np(RelayBPDecoder(w.H, w.priors, **{**RELAY, "num_sets": k}).decode(syn))
        fracs.append(float((o["found_count"] < S).mean()))
    # a shot gains at most one solution per leg, so the fraction is 1 until leg S-1
    k0 = next(k for k, f in enumerate(fracs) if f < 1.0)
    k1 = next(k for k in range(k0 + 1, len(fracs)) if 0.0 < fracs[k] < fracs[k0])
    thr = (fracs[k1 - 1] + fracs[k1]) / 2
    stop = next(k for k, f in enumerate(fracs) if f < thr)
    assert stop == k1
    ref = _np(RelayBPDecoder(w.H, w.priors, **{**RELAY, "num_sets": stop}).decode(syn))
    got = RelayBPDecoder(w.H, w.priors, fast_max_unconverged_pct=thr, **RELAY).decode(syn)
    _same(_np(got), ref)
    unc = got["unconverged_indices"].cpu().numpy()
    assert len(unc) > 0
    np.testing.assert_array_equal(unc, np.nonzero(ref["found_count"] < S)[0])


# --- unconverged correction, on a small random code whose random syndromes often have no solution


def _problem(C=24, V=40, deg=4, seed=7):
    rng = np.random.default_rng(seed)
    H = np.zeros((C, V), np.uint8)
    for c in range(C):
        H[c, rng.choice(V, deg, replace=False)] = 1
    return csr_matrix(H)


def _syn(B, C, seed=3):
    return torch.from_numpy(np.random.default_rng(seed).integers(0, 2, size=(B, C)).astype(np.uint8)).to(DEV)


def _small(H, syn, num_sets, **kw):
    kw.setdefault("pre_iter", 4)
    dec = RelayBPDecoder(H, np.full(H.shape[1], 0.06), num_sets=num_sets, set_max_iter=4, gamma0=0.1,
                         stop_nconv=1, device=[0], seed=42, algo="relay", **kw)
    return _np(dec.decode(syn))


def test_unconverged_shot_returns_leg0_hard_decision():
    H = _problem()
    syn = _syn(512, H.shape[0])
    full, leg0 = _small(H, syn, 3), _small(H, syn, 0)
    never = full["found_count"] == 0
    assert never.sum() > 0
    np.testing.assert_array_equal(full["errors"][never], leg0["errors"][never])


def test_early_exit_unconverged_shot_returns_leg0_hard_decision():
    H = _problem()
    syn = _syn(512, H.shape[0])
    leg0, leg1 = _small(H, syn, 0), _small(H, syn, 1)
    u0, u1 = float((leg0["found_count"] == 0).mean()), float((leg1["found_count"] == 0).mean())
    assert u1 < u0
    dec = RelayBPDecoder(H, np.full(H.shape[1], 0.06), num_sets=3, set_max_iter=4, gamma0=0.1, stop_nconv=1,
                         device=[0], seed=42, algo="relay", pre_iter=4, fast_max_unconverged_pct=(u0 + u1) / 2)
    full = _np(dec.decode(syn))
    assert len(full["unconverged_indices"]) > 0
    never = full["found_count"] == 0
    assert never.sum() > 0
    np.testing.assert_array_equal(full["errors"][never], leg0["errors"][never])
    _same(full, leg1, ("errors", "found_count", "iterations", "valid_mask"))


def test_pre_iter_zero_returns_relay_leg1_hard_decision():
    H = _problem()
    syn = _syn(512, H.shape[0])
    full = _small(H, syn, 3, pre_iter=0)
    leg1 = _small(H, syn, 1, pre_iter=0, unconverged_correction="last_leg")
    never = full["found_count"] == 0
    assert never.sum() > 0
    np.testing.assert_array_equal(full["errors"][never], leg1["errors"][never])
    assert full["errors"][never].any(axis=1).any()


def test_converged_shots_satisfy_the_syndrome():
    H = _problem()
    syn = _syn(512, H.shape[0])
    full = _small(H, syn, 3)
    ok = full["found_count"] > 0
    assert ok.sum() > 0
    e = full["errors"][ok].astype(np.int64)
    np.testing.assert_array_equal((H @ e.T % 2).T, syn.cpu().numpy()[ok])


def test_last_leg_returns_final_hard_decision():
    """last_leg: an unconverged shot returns the hard decision after the last leg, which for a
    decode stopped early is the hard decision after the leg it stopped on."""
    H = _problem()
    syn = _syn(512, H.shape[0])
    full = _small(H, syn, 3, unconverged_correction="last_leg")
    dec = RelayBPDecoder(H, np.full(H.shape[1], 0.06), num_sets=3, set_max_iter=4, gamma0=0.1, stop_nconv=1,
                         device=[0], seed=42, algo="relay", pre_iter=4, unconverged_correction="last_leg")
    st = dec.new_state(syn.shape[0])
    dec.decode_phases(syn, suspend=st, legs_end=1)
    got = _np(dec.decode_phases(syn, resume=st, legs_begin=1))
    _same(got, full, ("errors", "found_count", "iterations"))
