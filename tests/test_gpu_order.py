"""Queue order of the persistent decode kernel (B200).

``rbp_batch.shot_order`` only changes which shot a group takes next, so the
outputs must not depend on it; the default relay decode of large batches runs
the pre-iterations first and then queues the shots they left unconverged
first (``hard_shots_first``), which must give exactly the single-launch result.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from pelagos_b200 import RelayBPDecoder, codes
from pelagos_b200 import _native as nat
from pelagos_b200.decoder import _ptr

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)
KEYS = ("errors", "found_count", "iterations", "weight_fixed", "valid_mask", "weights", "unconverged_indices")


def _np(out):
    return {k: v.cpu().numpy() for k, v in out.items() if isinstance(v, torch.Tensor)}


@pytest.fixture(scope="module")
def shots():
    w = codes.workload("bb144_phen", p=0.004)
    return w, torch.from_numpy(w.sample(8192, seed=123)[1]).to(DEV)


@pytest.mark.parametrize("kw", [{}, {"gamma_draw": "per_row"}, {"data_type": "bfloat16"},
                                {"unconverged_correction": "last_leg"}])
def test_hard_first_equals_single_launch(shots, kw):
    w, syn = shots
    a = RelayBPDecoder(w.H, w.priors, hard_shots_first=True, **RELAY, **kw)
    b = RelayBPDecoder(w.H, w.priors, hard_shots_first=False, **RELAY, **kw)
    oa = _np(a.decode(syn, return_last_posterior=True))
    ob = _np(b.decode(syn, return_last_posterior=True))
    assert (ob["iterations"] > RELAY["pre_iter"] + 4 * RELAY["set_max_iter"]).any(), "no hard shot in the sample"
    for k in KEYS + ("last_posterior",):
        np.testing.assert_array_equal(oa[k], ob[k], err_msg=k)


def test_explicit_orders_do_not_change_results(shots):
    w, syn = shots
    syn = syn[:2048].contiguous()
    dec = RelayBPDecoder(w.H, w.priors, hard_shots_first=False, **RELAY)
    ref = _np(dec.decode(syn))
    B = syn.shape[0]
    gid = dec.device_ids[0]
    stream = torch.cuda.current_stream().cuda_stream
    for order in (torch.arange(B - 1, -1, -1), torch.randperm(B, generator=torch.Generator().manual_seed(3))):
        order = order.to(device=DEV, dtype=torch.int32)
        found = torch.full((B,), -7, dtype=torch.int32, device=DEV)
        iters = torch.empty(B, dtype=torch.int32, device=DEV)
        errs = torch.empty(B, dec.V, dtype=torch.uint8, device=DEV)
        wfix = torch.empty(B, dtype=torch.int64, device=DEV)
        bi = nat.RbpBatch(syndromes=_ptr(syn), gamma0=float(np.float32(dec.gamma0)), pre_iter=dec.pre_iter,
                          shot_order=_ptr(order))
        bo = nat.RbpOutputs(errors=_ptr(errs), weight_fixed=_ptr(wfix), found_count=_ptr(found),
                            iterations=_ptr(iters))
        dec._native[gid].decode(B, bi, bo, stream)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(found.cpu().numpy(), ref["found_count"])
        np.testing.assert_array_equal(iters.cpu().numpy(), ref["iterations"])
        np.testing.assert_array_equal(errs.cpu().numpy(), ref["errors"])
        np.testing.assert_array_equal(wfix.cpu().numpy(), ref["weight_fixed"])


def test_out_of_range_order_entries_are_skipped(shots):
    w, syn = shots
    syn = syn[:512].contiguous()
    dec = RelayBPDecoder(w.H, w.priors, hard_shots_first=False, **RELAY)
    ref = _np(dec.decode(syn))
    B = syn.shape[0]
    order = torch.arange(B, dtype=torch.int32)
    order[3] = -1
    order[10] = B + 5
    order = order.to(DEV)
    found = torch.full((B,), -7, dtype=torch.int32, device=DEV)
    iters = torch.full((B,), -7, dtype=torch.int32, device=DEV)
    bi = nat.RbpBatch(syndromes=_ptr(syn), gamma0=float(np.float32(dec.gamma0)), pre_iter=dec.pre_iter,
                      shot_order=_ptr(order))
    bo = nat.RbpOutputs(found_count=_ptr(found), iterations=_ptr(iters))
    dec._native[dec.device_ids[0]].decode(B, bi, bo, torch.cuda.current_stream().cuda_stream)
    f = found.cpu().numpy()
    assert f[3] == -7 and f[10] == -7          # shots 3 and 10 were never taken
    keep = np.ones(B, bool)
    keep[[3, 10]] = False
    np.testing.assert_array_equal(f[keep], ref["found_count"][keep])


def test_cuda_graph_replay_equals_eager_decode(shots):
    """cuda_graph=True: one graph replay per call gives the eager result for every batch of the
    captured size (the input is copied in, the results cloned out), host syndromes included, and
    a launch-shape change recaptures."""
    w, syn = shots
    eager = RelayBPDecoder(w.H, w.priors, **RELAY)
    graphed = RelayBPDecoder(w.H, w.priors, cuda_graph=True, **RELAY)
    a, b = syn[:4096].contiguous(), syn[4096:].contiguous()
    want_a, want_b = _np(eager.decode(a)), _np(eager.decode(b))
    got_a = graphed.decode(a)
    got_b = graphed.decode(b.cpu())           # host syndromes: copied into the graph's input
    got_a2 = _np(graphed.decode(a))
    assert len(graphed._cuda_graphs) == 1
    for got, want in ((_np(got_a), want_a), (_np(got_b), want_b), (got_a2, want_a)):
        for k in KEYS:
            np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    graphed.configure_launch(704, 1, 1)
    got = _np(graphed.decode(b))
    assert graphed._cuda_graphs[4096][0][1] == (704, 1, 1, 0)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], want_b[k], err_msg=k)
