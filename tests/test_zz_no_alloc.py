"""rbp_decode_static: the decode entry point that allocates nothing.

Callers such as a real-time decoding service with a fixed device-memory budget
cannot allocate device memory between syndrome rounds (an allocation
synchronises the device and its latency is unbounded), and a process whose
device memory is already reserved by another allocator may see allocations
fail.  For them the library's derived graph tables and the kernel's work
counter live in a static device array instead of cudaMalloc'd buffers.

These tests call that entry point through the C ABI and check, on two calls
in a row, that its outputs are identical to those of the existing entry point
(rbp_decode, reached through RelayBPDecoder): the bit-exact bar of every other
parity test in this suite.  The file is collected last so that a failure here
leaves every other test already run.
"""

from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest
import torch

from pelagos_b200 import RelayBPDecoder, codes
from pelagos_b200 import _native as nat

pytestmark = pytest.mark.gpu

DEV = "cuda:0"
RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)


def _ptr(t):
    return ct.c_void_p(t.data_ptr()) if t is not None else ct.c_void_p(0)


def _static_decode(dec: RelayBPDecoder, syn: torch.Tensor) -> dict:
    """One rbp_decode_static call with the decoder's graph, priors, leg table and (for
    normalized min-sum) its per-iteration alpha table, all in device memory."""
    from pelagos_b200.utils import alpha_schedule

    g = dec.graph
    B = int(syn.shape[0])
    llr = torch.from_numpy(dec.log_prior_ratios).to(DEV)
    legs = torch.from_numpy(np.ascontiguousarray(dec._leg_table(0))).to(DEV)
    use_alpha, alpha = alpha_schedule(dec.normalized_min_sum_alpha, dec.alpha_iteration_scaling_factor,
                                      max(dec.pre_iter, dec.set_max_iter, 1))
    alpha_dev = torch.from_numpy(np.ascontiguousarray(alpha, np.float32)).to(DEV) if use_alpha else None
    post_dtype = torch.float64 if dec.dtype_str == "float64" else torch.float32
    out = {
        "errors": torch.full((B, dec.V), 7, dtype=torch.uint8, device=DEV),
        "weight_fixed": torch.zeros(B, dtype=torch.int64, device=DEV),
        "found_count": torch.full((B,), -1, dtype=torch.int32, device=DEV),
        "iterations": torch.full((B,), -1, dtype=torch.int32, device=DEV),
        "last_posterior": torch.full((B, dec.V), float("nan"), dtype=post_dtype, device=DEV),
    }
    batch = nat.RbpBatch(syndromes=_ptr(syn), llr_per_shot=None, gamma_pre=None,
                         gamma0=float(np.float32(dec.gamma0)), init_posterior=None, gamma_legs_shot=None,
                         n_shot_legs=0, pre_iter=dec.pre_iter, skip_relay_legs=0)
    outs = nat.RbpOutputs(errors=_ptr(out["errors"]), errors_packed=None, weights=None,
                          weight_fixed=_ptr(out["weight_fixed"]), found_count=_ptr(out["found_count"]),
                          iterations=_ptr(out["iterations"]), last_posterior=_ptr(out["last_posterior"]))
    params = dec._params()
    rc = nat.lib().rbp_decode_static(
        g.C, g.V, g.E, nat.i32_ptr(g.chk_ptr), nat.i32_ptr(g.edge_var), nat.i32_ptr(g.var_ptr),
        nat.i32_ptr(g.var_edges), ct.byref(params), _ptr(llr), _ptr(legs), _ptr(alpha_dev),
        int(alpha_dev.numel()) if alpha_dev is not None else 0, 0, B,
        ct.byref(batch), ct.byref(outs), ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == nat.RBP_OK, nat.lib().rbp_last_error().decode()
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def _decoder_entry(dec: RelayBPDecoder, syn: torch.Tensor) -> dict:
    out = dec.decode(syn, return_last_posterior=True)
    torch.cuda.synchronize()
    return {k: out[k].cpu().numpy() for k in ("errors", "weight_fixed", "found_count", "iterations",
                                                 "last_posterior")}


def _assert_identical(got: dict, want: dict) -> None:
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


@pytest.mark.parametrize("workload,shots,extra", [
    ("bb144_phen", 2048, {}),
    ("bb72_cc", 1024, {}),
    ("bb144_phen", 512, {"data_type": "float16"}),
    ("bb144_phen", 512, {"data_type": "bfloat16"}),
    ("bb72_cc", 512, {"data_type": "float64"}),
    ("bb72_cc", 512, {"normalized_min_sum_alpha": 0.0}),   # alpha ramp: the alpha table is read per iteration
    ("bb72_cc", 512, {"normalized_min_sum_alpha": 0.8, "data_type": "float16"}),
])
def test_static_entry_matches_decoder_entry_on_two_calls(workload, shots, extra):
    """Every message type's slot layout and the caller-supplied alpha table, against rbp_decode."""
    w = codes.workload(workload)
    err, syn = w.sample(shots, seed=99)
    syn = torch.from_numpy(syn).to(DEV)
    dec = RelayBPDecoder(w.H, w.priors, **{**RELAY, **extra})
    want = _decoder_entry(dec, syn)
    first = _static_decode(dec, syn)
    second = _static_decode(dec, syn)   # the array keeps the first call's contents
    _assert_identical(first, want)
    _assert_identical(second, want)


def test_static_entry_rewrites_tables_between_graphs():
    """A call with another graph replaces every table the previous call left."""
    a, b = codes.workload("bb144_phen"), codes.workload("bb72_cc")
    sa = torch.from_numpy(a.sample(512, seed=5)[1]).to(DEV)
    sb = torch.from_numpy(b.sample(512, seed=6)[1]).to(DEV)
    da = RelayBPDecoder(a.H, a.priors, **RELAY)
    db = RelayBPDecoder(b.H, b.priors, **RELAY)
    _assert_identical(_static_decode(da, sa), _decoder_entry(da, sa))
    _assert_identical(_static_decode(db, sb), _decoder_entry(db, sb))
    _assert_identical(_static_decode(da, sa), _decoder_entry(da, sa))


def test_static_entry_rejects_tables_beyond_the_array():
    """65,535 variables with a degree-8 variable need 2 * 8 * 65,535 bytes of slot table alone."""
    V, C = 65535, 8
    chk_ptr = np.arange(C + 1, dtype=np.int32)          # 8 checks, one edge each
    edge_var = np.zeros(C, dtype=np.int32)               # all on variable 0 (degree 8)
    var_ptr = np.full(V + 1, C, dtype=np.int32)
    var_ptr[0] = 0
    var_edges = np.arange(C, dtype=np.int32)
    params = nat.RbpParams(pre_iter=1, num_sets=0, set_max_iter=1, stop_nconv=1, msg_type=nat.RBP_MSG_F32)
    llr = torch.zeros(V, dtype=torch.float32, device=DEV)
    syn = torch.zeros(1, C, dtype=torch.uint8, device=DEV)
    found = torch.zeros(1, dtype=torch.int32, device=DEV)
    iters = torch.zeros(1, dtype=torch.int32, device=DEV)
    batch = nat.RbpBatch(syndromes=_ptr(syn), pre_iter=1)
    outs = nat.RbpOutputs(found_count=_ptr(found), iterations=_ptr(iters))
    rc = nat.lib().rbp_decode_static(C, V, C, nat.i32_ptr(chk_ptr), nat.i32_ptr(edge_var), nat.i32_ptr(var_ptr),
                                     nat.i32_ptr(var_edges), ct.byref(params), _ptr(llr), None, None, 0, 0, 1,
                                     ct.byref(batch), ct.byref(outs), None)
    assert rc == nat.RBP_ERR_UNSUPPORTED
    msg = nat.lib().rbp_last_error().decode()
    assert "scratch" in msg and str(nat.STATIC_SCRATCH_BYTES) in msg


def test_static_entry_refuses_a_capturing_stream():
    """The tables are staged from host memory that is gone by the time a graph replays, so a
    call on a stream under capture is refused before anything is enqueued."""
    w = codes.workload("bb72_cc")
    syn = torch.from_numpy(w.sample(64, seed=3)[1]).to(DEV)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    _static_decode(dec, syn)  # first call on the device: looks up the array's address
    g = dec.graph
    found = torch.zeros(64, dtype=torch.int32, device=DEV)
    iters = torch.zeros(64, dtype=torch.int32, device=DEV)
    llr = torch.from_numpy(dec.log_prior_ratios).to(DEV)
    legs = torch.from_numpy(np.ascontiguousarray(dec._leg_table(0))).to(DEV)
    batch = nat.RbpBatch(syndromes=_ptr(syn), gamma0=float(np.float32(dec.gamma0)), pre_iter=dec.pre_iter)
    outs = nat.RbpOutputs(found_count=_ptr(found), iterations=_ptr(iters))
    params = dec._params()
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        graph.capture_begin()
        rc = nat.lib().rbp_decode_static(
            g.C, g.V, g.E, nat.i32_ptr(g.chk_ptr), nat.i32_ptr(g.edge_var), nat.i32_ptr(g.var_ptr),
            nat.i32_ptr(g.var_edges), ct.byref(params), _ptr(llr), _ptr(legs), None, 0, 0, 64,
            ct.byref(batch), ct.byref(outs), ct.c_void_p(side.cuda_stream))
        found.add_(1)  # something for the graph to hold
        graph.capture_end()
    assert rc == nat.RBP_ERR_UNSUPPORTED
    assert "captured" in nat.lib().rbp_last_error().decode()
    graph.replay()
    torch.cuda.synchronize()
    assert int(found.sum()) == 64  # the capture itself was left intact: one recorded add
