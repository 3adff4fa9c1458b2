"""Parity at the benchmark's own size and schedule (B200).

The benchmark batch itself — 65,536 seeded shots of the [[144,12,12]]
phenomenological workload at p = 0.003 (seed 2026), full Relay-BP-S schedule
(pre 80, 100 legs x 60, gamma0 0.65, U(-0.24, 0.66), stop_nconv 5), float32 —
decoded on the GPU and compared bit for bit with the CPU oracle:

* the plain decoder (RelayBPDecoder.decode), with every kernel family (the
  block-per-group kernel with one and with two shots per group, the kernel
  whose blocks hold several one-shot groups, and one-shot groups at two
  resident blocks per SM with 352 and with 448 threads, the latter the
  benchmark's committed shape);
* the gated learned decoder (LearnedRelayBPDecoder, gate=True) against the
  oracle's per-shot emulation of it: shots the pre-iterations solved run relay
  legs 0-3 at the constant top strength, the others run them with the
  network's strengths (one row per shot), and every shot the seeded table
  after that.

The oracle runs in chunks over every host core (a few seconds per batch).
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
SHOTS, SEED, P = 65536, 2026, 0.003
CHUNK = 8192


@pytest.fixture(scope="module")
def bench_batch():
    w = codes.workload("bb144_phen", p=P)
    err, syn = w.sample(SHOTS, seed=SEED)
    return w, syn


def _oracle_chunks(dec, syn, legs, gamma_legs_shot=None, idx=None):
    """Oracle outputs for syn[idx] (all shots when idx is None), chunk by chunk, without the posteriors."""
    g = O.reference_graph(dec.H_csr)
    idx = np.arange(len(syn)) if idx is None else idx
    out = {k: [] for k in KEYS}
    for s in range(0, len(idx), CHUNK):
        sel = idx[s:s + CHUNK]
        gls = None if gamma_legs_shot is None else gamma_legs_shot[s:s + CHUNK]
        r = O.decode(g, syn[sel], dec.log_prior_ratios, pre_iter=dec.pre_iter, num_sets=dec.num_sets,
                     set_max_iter=dec.set_max_iter, stop_nconv=dec.stop_nconv, gamma0=dec.gamma0, gamma_legs=legs,
                     gamma_legs_shot=gls)
        for k in KEYS:
            out[k].append(r[k])
    return {k: np.concatenate(v) for k, v in out.items()}


def _assert_same(got, want, what):
    for k in KEYS:
        a, b = got[k], want[k]
        if not np.array_equal(a, b):
            bad = np.nonzero((a != b).reshape(len(a), -1).any(1))[0]
            raise AssertionError(f"{what}: {k} differs on {len(bad)} of {len(a)} shots, first {bad[:8].tolist()}")


@pytest.fixture(scope="module")
def plain_oracle(bench_batch):
    w, syn = bench_batch
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    return _oracle_chunks(dec, syn, dec._leg_table(0))


@pytest.mark.parametrize("launch", [(0, 1, 1), (0, 1, 2), (0, 0, 1), (352, 1, 1, 2), (448, 1, 1, 2)])
def test_plain_decode_of_the_bench_batch_matches_oracle(bench_batch, plain_oracle, launch):
    w, syn = bench_batch
    dec = RelayBPDecoder(w.H, w.priors, launch=launch, **RELAY)
    out = dec.decode(torch.from_numpy(syn).to(DEV))
    got = {k: out[k].cpu().numpy() for k in KEYS}
    _assert_same(got, plain_oracle, f"plain decode, launch {launch}")
    # the long relay tails are exercised
    assert got["iterations"].max() > 200


@pytest.mark.parametrize("launch", [(0, 1, 1), (0, 1, 2), (0, 0, 1), (352, 1, 1, 2), (448, 1, 1, 2)])
def test_gated_learned_decode_of_the_bench_batch_matches_oracle_emulation(bench_batch, launch):
    from pelagos_b200.proposal import LearnedRelayBPDecoder, ProposalNet, default_weights_path, load_params

    w, syn = bench_batch
    dec = RelayBPDecoder(w.H, w.priors, launch=launch, **RELAY)
    net = ProposalNet(dec, load_params(default_weights_path("bb144_phen", P))[0])
    learned = LearnedRelayBPDecoder(dec, net, learned_legs=4, gate=True, graph=False)
    syn_d = torch.from_numpy(syn).to(DEV)
    out = learned.decode(syn_d)
    got = {k: out[k].cpu().numpy() for k in KEYS}

    # the emulation: which shots the pre-iterations solve, and the network's strengths for the others
    pre = dec.decode_phases(syn_d, skip_relay_legs=True, return_last_posterior=True)
    solved = pre["found_count"].cpu().numpy() > 0
    uns = np.nonzero(~solved)[0]
    assert 0 < len(uns) < SHOTS // 20
    lo, hi = (float(x) for x in RELAY["gamma_dist_interval"])
    gam = net.propose(syn_d[uns], pre["last_posterior"][uns], lo, hi).cpu().numpy()
    legs = dec._leg_table(0)
    legs_solved = legs.copy()
    legs_solved[:4] = np.float32(hi)  # solved shots: the constant top strength on legs 0-3
    want = {k: np.empty_like(v) for k, v in got.items()}
    sol = np.nonzero(solved)[0]
    r_sol = _oracle_chunks(dec, syn, legs_solved, idx=sol)
    r_uns = _oracle_chunks(dec, syn, legs, gamma_legs_shot=np.repeat(gam[:, None, :], 4, axis=1), idx=uns)
    for k in KEYS:
        want[k][sol] = r_sol[k]
        want[k][uns] = r_uns[k]
    _assert_same(got, want, f"gated learned decode, launch {launch}")
