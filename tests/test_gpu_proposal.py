"""Learned relay-leg proposal on the B200: the network's CUDA kernels against the
CPU specification (oracle/proposal_oracle.py), and the learned decode against
the decoder oracle's per-shot emulation.

* the training-path forward and the tensor-core inference kernel against the
  float64 specification (same bf16 rounding points; fp32 sums);
* the gradients of the training step against the specification's backward,
  which is itself checked against finite differences on the CPU;
* one and two AdamW steps against the specification's AdamW;
* the learned decode = the CPU decoder oracle run with the proposed strengths
  as per-shot rows of legs 0-3 and the seeded table after (bit for bit);
* training lowers the loss.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import oracle as O
from oracle import proposal_oracle as po
from pelagos_b200 import RelayBPDecoder, codes
from pelagos_b200.proposal import (RELAY, LearnedRelayBPDecoder, ProposalNet, ShotSampler, TrainConfig, init_params,
                                   make_tuples, train)

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def setup():
    w = codes.workload("bb144_phen", p=0.004)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    err, syn = w.sample(64, seed=5)
    err_d, syn_d = torch.from_numpy(err).to(DEV), torch.from_numpy(syn).to(DEV)
    post, target = make_tuples(dec, syn_d, err_d)
    theta = init_params(3) + np.random.default_rng(4).normal(0, 0.05, 4805).astype(np.float32)
    net = ProposalNet(dec, theta)
    g = po.Graph.from_csr(w.H)
    return dict(w=w, dec=dec, err=err, syn=syn, syn_d=syn_d, post=post, target=target, theta=theta, net=net, g=g,
                llr=dec.log_prior_ratios)


def _close(a, b, what, atol, mean_tol):
    d = np.abs(a - b)
    assert d.max() <= atol, f"{what}: max |diff| {d.max():.3g} at {np.unravel_index(d.argmax(), d.shape)}"
    assert d.mean() <= mean_tol, f"{what}: mean |diff| {d.mean():.3g}"


def test_init_params_match_specification():
    np.testing.assert_array_equal(init_params(0), po.init_params(0))


def test_forward_matches_specification(setup):
    s = setup
    B = 6
    ref = po.forward(s["theta"], s["g"], s["syn"][:B], s["post"][:B].cpu().numpy(), s["llr"])
    got = s["net"].forward(s["syn_d"][:B], s["post"][:B]).cpu().numpy()
    # fp32 vs float64 sums; a bf16 rounding that lands on the other side of a tie moves one input by 2^-8
    _close(got, ref, "training forward", atol=2e-2, mean_tol=2e-4)


def test_inference_kernel_matches_specification_and_training_forward(setup):
    s = setup
    B = 6
    ref = po.forward(s["theta"], s["g"], s["syn"][:B], s["post"][:B].cpu().numpy(), s["llr"])
    gam, r = s["net"].propose(s["syn_d"], s["post"], -0.24, 0.66, logits=True)
    r = r.cpu().numpy()
    _close(r[:B], ref, "tensor-core inference", atol=2e-2, mean_tol=2e-4)
    fwd = s["net"].forward(s["syn_d"], s["post"]).cpu().numpy()
    _close(r, fwd, "inference vs training forward", atol=2e-2, mean_tol=1e-4)
    gam = gam.cpu().numpy()
    np.testing.assert_allclose(gam, -0.24 + 0.9 / (1 + np.exp(-r)), rtol=0, atol=2e-6)
    assert (gam > -0.24).all() and (gam < 0.66).all()


def test_gradients_match_specification(setup):
    s = setup
    B = 6
    cfg = TrainConfig(w_neg=20.0)
    grads = torch.zeros(4805, device=DEV)
    loss = torch.zeros(1, device=DEV)
    s["net"].set_params(s["theta"])
    s["net"].train_step(s["syn_d"][:B], s["post"][:B], s["target"][:B], cfg, lr=0.0, loss_out=loss, grads_out=grads)
    L, ref = po.backward(s["theta"], s["g"], s["syn"][:B], s["post"][:B].cpu().numpy(), s["llr"],
                         s["target"][:B].cpu().numpy(), w_neg=20.0)
    assert float(loss) == pytest.approx(L, rel=1e-4)
    got = grads.cpu().numpy()
    for name, (o, shape) in po.offsets().items():
        n = int(np.prod(shape))
        a, b = got[o:o + n], ref[o:o + n]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 2e-3, f"{name}: relative gradient error {err:.3g}"
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-3


def test_adamw_steps_match_specification(setup):
    s = setup
    B = 6
    cfg = TrainConfig(weight_decay=0.01)
    net = s["net"]
    net.set_params(s["theta"])
    theta = s["theta"].astype(np.float64)
    m = np.zeros_like(theta)
    v = np.zeros_like(theta)
    grads = torch.zeros(4805, device=DEV)
    for step, lr in ((1, 3e-3), (2, 1e-3)):
        net.train_step(s["syn_d"][:B], s["post"][:B], s["target"][:B], cfg, lr=lr, grads_out=grads)
        theta, m, v = po.adamw(theta, m, v, grads.cpu().numpy().astype(np.float64), step, lr,
                               beta1=cfg.beta1, beta2=cfg.beta2, eps=cfg.eps, wd=cfg.weight_decay)
        np.testing.assert_allclose(net.params().cpu().numpy(), theta, rtol=1e-5, atol=1e-7)
    net.set_params(s["theta"])


def test_learned_decode_matches_oracle_emulation(setup):
    """Each shot's learned decode equals the CPU decoder oracle run on that shot with the
    proposed strengths as its rows for legs 0-3 and the seeded table for the rest."""
    s = setup
    dec, net = s["dec"], s["net"]
    net.set_params(s["theta"])
    learned = LearnedRelayBPDecoder(dec, net, learned_legs=4)
    out = {k: v.cpu().numpy() for k, v in learned.decode(s["syn_d"]).items()}
    gam = net.propose(s["syn_d"], s["post"], -0.24, 0.66).cpu().numpy()
    rows = np.repeat(gam[:, None, :], 4, axis=1)
    g = O.reference_graph(dec.H_csr)
    ref = O.decode(g, s["syn"], dec.log_prior_ratios, pre_iter=dec.pre_iter, num_sets=dec.num_sets,
                   set_max_iter=dec.set_max_iter, stop_nconv=dec.stop_nconv, gamma0=dec.gamma0,
                   gamma_legs=dec._leg_table(0), gamma_legs_shot=rows)
    for k in ("errors", "found_count", "iterations", "weight_fixed", "valid_mask"):
        np.testing.assert_array_equal(out[k], ref[k], err_msg=k)
    H = s["w"].H
    ok = out["found_count"] > 0
    np.testing.assert_array_equal((H @ out["errors"][ok].T.astype(np.int64) % 2).T, s["syn"][ok])


@pytest.mark.parametrize("fused", [False, True])
def test_gated_decode_matches_oracle_emulation(setup, fused):
    """gate=True: shots the pre-iterations solved get the top strength on legs 0-3, the others the
    network's proposal; each equals the oracle run with those rows."""
    s = setup
    w = codes.workload("bb144_phen", p=0.006)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    syn = w.sample(768, seed=9)[1]
    syn_d = torch.from_numpy(syn).to(DEV)
    net = ProposalNet(dec, s["theta"])
    learned = LearnedRelayBPDecoder(dec, net, gate=True, fused=fused)
    out = {k: v.cpu().numpy() for k, v in learned.decode(syn_d).items()}
    pre = dec.decode_phases(syn_d, skip_relay_legs=True, return_last_posterior=True)
    solved = pre["found_count"].cpu().numpy() > 0
    assert solved.any() and (~solved).any()
    gam = net.propose(syn_d, pre["last_posterior"], -0.24, 0.66).cpu().numpy()
    gam[solved] = np.float32(0.66)
    rows = np.repeat(gam[:, None, :], 4, axis=1)
    ref = O.decode(O.reference_graph(dec.H_csr), syn, dec.log_prior_ratios, pre_iter=dec.pre_iter,
                   num_sets=dec.num_sets, set_max_iter=dec.set_max_iter, stop_nconv=dec.stop_nconv,
                   gamma0=dec.gamma0, gamma_legs=dec._leg_table(0), gamma_legs_shot=rows)
    for k in ("errors", "found_count", "iterations", "weight_fixed", "valid_mask"):
        np.testing.assert_array_equal(out[k], ref[k], err_msg=k)


def test_graph_replay_equals_eager(setup):
    """The captured learned decode gives the eager results, on refilled inputs too."""
    s = setup
    w = codes.workload("bb144_phen", p=0.005)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    net = ProposalNet(dec, s["theta"])
    eager = LearnedRelayBPDecoder(dec, net, gate=True, graph=False)
    graphed = LearnedRelayBPDecoder(dec, net, gate=True, graph=True)
    for seed in (21, 22):
        syn = torch.from_numpy(w.sample(2048, seed=seed)[1]).to(DEV)
        a = {k: v.cpu().numpy() for k, v in eager.decode(syn).items()}
        b = {k: v.cpu().numpy() for k, v in graphed.decode(syn).items()}
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_decode_stream_equals_decode(setup):
    """The overlapped stream of host batches returns, batch by batch, what decode() returns,
    into a ring of two pinned host buffer sets and into freshly allocated ones."""
    s = setup
    w = codes.workload("bb144_phen", p=0.005)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    net = ProposalNet(dec, s["theta"])
    learned = LearnedRelayBPDecoder(dec, net, gate=True)
    batches = [torch.from_numpy(w.sample(2048, seed=40 + i)[1]).pin_memory() for i in range(5)]
    ref = [{k: v.cpu().numpy() for k, v in learned.decode(b).items()} for b in batches]
    keys = ("errors", "weight_fixed", "found_count", "iterations")
    got = learned.decode_stream(batches)
    for i in range(5):
        for k in keys:
            np.testing.assert_array_equal(got[i][k].numpy(), ref[i][k], err_msg=f"{k} of batch {i}")
    ring = [{k: torch.empty_like(v).pin_memory() for k, v in got[0].items()} for _ in range(2)]
    for i in range(5):
        out = learned.decode_stream(batches[: i + 1], out=[ring[j % 2] for j in range(i + 1)])
        for k in keys:
            np.testing.assert_array_equal(out[i][k].numpy(), ref[i][k], err_msg=f"{k} of batch {i} (ring)")
    with pytest.raises(ValueError):
        learned.decode_stream([batches[0].to(DEV)])


def test_training_lowers_the_loss(setup):
    s = setup
    cfg = TrainConfig(tuples=96 * 256, batch=256, lr=3e-3, lr_final=1e-3, log_every=32, seed=11)
    w = s["w"]
    net = ProposalNet(s["dec"], init_params(0))
    _, hist = train(s["dec"], w.H, w.priors, cfg, net=net, log=lambda *_: None)
    assert hist[-1]["loss"] < 0.7 * hist[0]["loss"], hist


def test_sampler_is_seeded(setup):
    w = setup["w"]
    a = ShotSampler(w.H, w.priors, DEV, 7).sample(128)
    b = ShotSampler(w.H, w.priors, DEV, 7).sample(128)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    e, syn = a
    np.testing.assert_array_equal((w.H @ e.cpu().numpy().T.astype(np.int64) % 2).T, syn.cpu().numpy())


def test_trained_network_gains_over_seeded_legs():
    """The committed network (trained on 2^22 decoder-generated tuples at p=0.003) against the
    method without it on 262,144 fresh seeded shots of the same workload: fewer iterations, no more
    logical failures, and more of the shots the pre-iterations leave unconverged solved than the
    constant-strength ablation solves."""
    from pelagos_b200.proposal import constant_params, default_weights_path, load_params

    w = codes.workload("bb144_phen", p=0.003)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    err, syn = w.sample(262144, seed=777001)
    syn_d = torch.from_numpy(syn).to(DEV)
    params, meta = load_params(default_weights_path("bb144_phen", 0.003))
    assert meta["train"]["tuples"] >= 1 << 22
    net = ProposalNet(dec, params)

    def run(fn):
        o = {k: v.cpu().numpy() for k, v in fn(syn_d).items() if isinstance(v, torch.Tensor)}
        conv = o["found_count"] > 0
        return o, int(w.logical_failures(err, o["errors"], conv).sum())

    plain, f_plain = run(dec.decode)
    gated, f_gated = run(LearnedRelayBPDecoder(dec, net, gate=True).decode)
    const, f_const = run(LearnedRelayBPDecoder(dec, ProposalNet(dec, constant_params())).decode)
    # the gate rule without the network: the solved shots' top strength, seeded legs for the rest
    rule, f_rule = run(LearnedRelayBPDecoder(dec, net, gate=True, network=False).decode)
    assert gated["iterations"].mean() < 0.75 * plain["iterations"].mean()
    assert f_gated <= f_plain and f_gated < f_const, (f_gated, f_plain, f_const)
    # what the network adds over the rule: the unconverged shots it solves
    assert f_gated < f_rule, (f_gated, f_rule)
    uns = (plain["found_count"] == 0) | (rule["found_count"] == 0)
    assert (gated["found_count"][uns] > 0).sum() > (rule["found_count"][uns] > 0).sum()
    ok = gated["found_count"] > 0
    np.testing.assert_array_equal((w.H @ gated["errors"][ok].T.astype(np.int64) % 2).T, syn[ok])


@pytest.mark.parametrize("dtype", ["bfloat16", "float16"])
def test_learned_decode_with_16_bit_messages(dtype):
    """The learned decode over a 16-bit-message decoder (float32 posteriors) matches the same
    decoder run with the proposed strengths as per-shot leg rows."""
    w = codes.workload("bb144_phen", p=0.005)
    dec = RelayBPDecoder(w.H, w.priors, data_type=dtype, **RELAY)
    from pelagos_b200.proposal import default_weights_path, load_params

    net = ProposalNet(dec, load_params(default_weights_path())[0])
    syn = torch.from_numpy(w.sample(2048, seed=31)[1]).to(DEV)
    out = {k: v.cpu().numpy() for k, v in LearnedRelayBPDecoder(dec, net, gate=False).decode(syn).items()}
    pre = dec.decode_phases(syn, skip_relay_legs=True, return_last_posterior=True)
    gam = net.propose(syn, pre["last_posterior"], -0.24, 0.66)
    ref = {k: v.cpu().numpy() for k, v in dec.decode(syn, leg_gammas=gam[:, None, :].expand(-1, 4, -1)).items()}
    for k in ("errors", "found_count", "iterations", "weight_fixed"):
        np.testing.assert_array_equal(out[k], ref[k], err_msg=k)
