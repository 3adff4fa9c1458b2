"""Mixed-code launches and the launch-shape autotuner (B200).

A mixed launch decodes several codes' batches in one persistent kernel; every
shot must come out exactly as when its own decoder decodes its batch alone
(the reference's batch-invariance contract, tests/test_decoder_fixes.py:184-268),
with or without CUDA-graph replay, and on repeated replays.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from pelagos_b200 import RelayBPDecoder, autotune, codes
from pelagos_b200.mixed import MixedDecoder

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)
KEYS = ("errors", "found_count", "iterations", "weight_fixed", "valid_mask")
MIX = [("bb72_cc", 0.03), ("bb144_cc", 0.03), ("bb144_phen", 0.003), ("ldpc2000", 0.02)]


def _np(out):
    return {k: v.cpu().numpy() for k, v in out.items() if isinstance(v, torch.Tensor)}


@pytest.fixture(scope="module")
def mixed_case():
    decs, syns = [], []
    for i, (name, p) in enumerate(MIX):
        w = codes.workload(name, p=p)
        decs.append(RelayBPDecoder(w.H, w.priors, **RELAY))
        syns.append(torch.from_numpy(w.sample(1536 + 512 * i, seed=40 + i)[1]).to(DEV))
    singles = [_np(d.decode(s)) for d, s in zip(decs, syns)]
    return decs, syns, singles


@pytest.mark.parametrize("graph", [False, True])
def test_mixed_launch_matches_separate_decodes(mixed_case, graph):
    decs, syns, singles = mixed_case
    mix = MixedDecoder(decs, graph=graph)
    for _ in range(2):  # a second decode (graph replay when captured)
        outs = [_np(o) for o in mix.decode(syns)]
        for name_p, o, ref in zip(MIX, outs, singles):
            for k in KEYS:
                np.testing.assert_array_equal(o[k], ref[k], err_msg=f"{name_p} {k}")
    info = mix.launch_info()
    assert len(info) == 4 and all(x["group_threads"] % 32 == 0 for x in info)


def test_mixed_launch_refills_and_reuses_buffers(mixed_case):
    """New syndromes in the same shapes reuse the captured graph; results follow the new inputs."""
    decs, syns, singles = mixed_case
    mix = MixedDecoder(decs, graph=True)
    mix.decode(syns)
    flipped = [torch.flip(s, dims=[0]) for s in syns]
    outs = [_np(o) for o in mix.decode(flipped)]
    for o, ref in zip(outs, singles):
        for k in ("errors", "found_count", "iterations"):
            np.testing.assert_array_equal(o[k], ref[k][::-1])


def test_autotune_keeps_results(tmp_path, monkeypatch):
    monkeypatch.setenv("PELAGOS_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    w = codes.workload("bb144_phen")
    syn = torch.from_numpy(w.sample(2048, seed=17)[1]).to(DEV)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    ref = _np(dec.decode(syn))
    shape = autotune.tune(dec, syn, shapes=[(256, 0), (512, 0), (864, 0), (448, 1, 2)], repeats=1)
    assert dec.launch_info()["group_threads"] == shape[0]
    got = _np(dec.decode(syn))
    for k in KEYS:
        np.testing.assert_array_equal(got[k], ref[k])
    assert autotune.lookup(dec, 2048) == shape  # cached
    dec2 = RelayBPDecoder(w.H, w.priors, **RELAY)
    assert autotune.tune(dec2, syn) == shape  # served from the cache


def test_mixed_launch_matches_oracle():
    """Each code's shots from one mixed launch, bit for bit against the CPU oracle (a few hundred
    shots per code; the oracle restates the reference loop per shot)."""
    from oracle import oracle as O

    decs, syns, hosts = [], [], []
    for i, (name, p) in enumerate(MIX):
        w = codes.workload(name, p=p)
        dec = RelayBPDecoder(w.H, w.priors, **RELAY)
        syn = w.sample(256, seed=70 + i)[1]
        decs.append(dec)
        syns.append(torch.from_numpy(syn).to(DEV))
        hosts.append(syn)
    outs = [_np(o) for o in MixedDecoder(decs, graph=True).decode(syns)]
    for (name, p), dec, syn, o in zip(MIX, decs, hosts, outs):
        ref = O.decode(O.reference_graph(dec.H_csr), syn, dec.log_prior_ratios, pre_iter=dec.pre_iter,
                       num_sets=dec.num_sets, set_max_iter=dec.set_max_iter, stop_nconv=dec.stop_nconv,
                       gamma0=dec.gamma0, gamma_legs=dec._leg_table(0))
        for k in ("errors", "found_count", "iterations", "weight_fixed"):
            np.testing.assert_array_equal(o[k], ref[k], err_msg=f"{name} {k}")


def test_mixed_autotune_keeps_results(mixed_case):
    """Per-code group sizes chosen by the mixed autotuner change no result."""
    decs, syns, singles = mixed_case
    mix = MixedDecoder(decs, graph=True)
    shapes = autotune.tune_mixed(mix, syns, repeats=1, rounds=1)
    assert [x["group_threads"] for x in mix.launch_info()] == shapes
    outs = [_np(o) for o in mix.decode(syns)]
    for name_p, o, ref in zip(MIX, outs, singles):
        for k in KEYS:
            np.testing.assert_array_equal(o[k], ref[k], err_msg=f"{name_p} {k}")
