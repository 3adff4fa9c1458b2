"""Learned relay-leg proposal: network, training on decoder-generated tuples, and
the learned decode (pre-iterations -> network -> relay legs).

The network (2-layer edge-conditioned message passing on the Tanner graph,
node width 64, message width 16, bf16 weights, fp32 sums) reads a shot's
syndrome and its posterior after the pre-iterations and proposes one memory
strength per variable for the first ``learned_legs`` relay legs.  Later legs
keep the decoder's seeded table, every decoded error must still satisfy
H e = s, and solutions are still ranked by the decoder's weight rule, so the
seeded legs remain the fallback.  The strengths reach the decoder as per-shot
leg gammas, the per-shot form of the reference's ``explicit_gammas`` rows
(src/pelagos/decoder.py:338-340, 481-491, 3685-3688), inside
``gamma_dist_interval``.

Training tuples come from the decoder itself.  For each seeded shot
(errors e ~ Bernoulli(priors), s = H e), the decoder runs the pre-iterations
and returns the posterior P; the target for variable v is y_v = [hard_v == e_v]
(the pre-iteration decision agrees with the true error), i.e. the converged-leg
strength hi where the carried posterior should be kept and lo where it should
be overruled.  The loss is the logistic loss of sigmoid(r_v) against y_v, with
weight ``w_neg`` on the (rare) variables whose decision is wrong.  Forward,
backward and AdamW run in the library's own CUDA kernels (rbp_net_*).
"""

from __future__ import annotations

import ctypes as ct
import json
import time
from dataclasses import asdict, dataclass
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _native as nat
from .decoder import RelayBPDecoder, _ptr

DATA_DIR = Path(__file__).resolve().parent / "data"

RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)


def param_count() -> int:
    n = ct.c_int64()
    nat.check(nat.lib().rbp_net_param_count(ct.byref(n)), "rbp_net_param_count")
    return int(n.value)


@dataclass
class TrainConfig:
    tuples: int = 1 << 22          # decoder-generated training tuples in total
    batch: int = 1024              # shots per step
    lr: float = 3e-3
    lr_final: float = 3e-4         # cosine decay to this
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    weight_decay: float = 1e-4
    w_neg: float = 20.0
    seed: int = 2024
    init_seed: int = 0
    log_every: int = 256


def init_params(seed: int = 0) -> np.ndarray:
    """Deterministic starting point (the same as the CPU specification's)."""
    rng = np.random.default_rng(seed)
    H, D, T, XC = 64, 16, 4, 6
    parts = [rng.normal(0, 1 / np.sqrt(XC), (H, XC))]
    for _ in (1, 2):
        parts += [rng.normal(0, 1 / np.sqrt(H), (D, H)), np.ones((T, D)) * 0.25,
                  rng.normal(0, 0.5 / np.sqrt(D), (H, D)), np.zeros(H)]
    parts += [rng.normal(0, 1 / np.sqrt(H), H) * 0.1, np.array([2.0, -2.0, -1.0, 0.0]), np.array([2.0])]
    out = np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)
    assert out.size == 4805
    return out


def load_params(path) -> tuple[np.ndarray, dict]:
    z = np.load(path, allow_pickle=False)
    return z["params"].astype(np.float32), json.loads(str(z["meta"]))


class ProposalNet:
    """Parameters and kernels of the proposal network on a decoder's graph and device."""

    def __init__(self, decoder: RelayBPDecoder, params=None):
        if decoder.num_gpus != 1:
            raise ValueError("the proposal network runs on one GPU")
        if decoder.dtype_str == "float64":
            raise ValueError("the proposal network reads float32 posteriors (float32/16-bit message decoders)")
        self.decoder = decoder
        gid = decoder.device_ids[0]
        self.device = torch.device(f"cuda:{gid}")
        self.n_params = param_count()
        self._h = ct.c_void_p()
        llr = np.ascontiguousarray(decoder.log_prior_ratios, dtype=np.float32)
        nat.check(nat.lib().rbp_net_create(decoder._native[gid]._graph, nat.f32_ptr(llr), ct.byref(self._h)),
                  "rbp_net_create")
        self.set_params(init_params(0) if params is None else params)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                nat.lib().rbp_net_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._h = ct.c_void_p()

    def _stream(self) -> ct.c_void_p:
        return ct.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def set_params(self, params) -> None:
        t = params if isinstance(params, torch.Tensor) else torch.from_numpy(np.asarray(params, np.float32))
        t = t.to(device=self.device, dtype=torch.float32).contiguous()
        if t.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {t.numel()}")
        nat.check(nat.lib().rbp_net_set_params(self._h, _ptr(t), self._stream()), "rbp_net_set_params")
        torch.cuda.current_stream(self.device).synchronize()

    def params(self) -> torch.Tensor:
        out = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        nat.check(nat.lib().rbp_net_get_params(self._h, _ptr(out), self._stream()), "rbp_net_get_params")
        return out

    def _inputs(self, syn, post):
        syn = syn.to(device=self.device, dtype=torch.uint8).contiguous()
        post = post.to(device=self.device, dtype=torch.float32).contiguous()
        if syn.ndim != 2 or syn.shape[1] != self.decoder.C or tuple(post.shape) != (syn.shape[0], self.decoder.V):
            raise ValueError("syndromes must be [B, C] and posteriors [B, V]")
        return syn, post

    def forward(self, syn: torch.Tensor, post: torch.Tensor) -> torch.Tensor:
        """Logits [B, V] from the training-path kernels (fp32 activations)."""
        syn, post = self._inputs(syn, post)
        out = torch.empty(syn.shape[0], self.decoder.V, dtype=torch.float32, device=self.device)
        nat.check(nat.lib().rbp_net_forward(self._h, syn.shape[0], _ptr(syn), _ptr(post), _ptr(out),
                                            self._stream()), "rbp_net_forward")
        return out

    def propose(self, syn: torch.Tensor, post: torch.Tensor, lo: float, hi: float, logits: bool = False):
        """Per-variable strengths [B, V] in (lo, hi) from the tensor-core inference kernel
        (and the logits when ``logits``)."""
        syn, post = self._inputs(syn, post)
        B = syn.shape[0]
        g = torch.empty(B, self.decoder.V, dtype=torch.float32, device=self.device)
        r = torch.empty_like(g) if logits else None
        nat.check(nat.lib().rbp_net_propose(self._h, B, _ptr(syn), _ptr(post), 0, float(lo), float(hi), None, None,
                                            _ptr(g), _ptr(r), self._stream()), "rbp_net_propose")
        return (g, r) if logits else g

    def propose_into(self, B: int, syn: torch.Tensor, post, lo: float, hi: float,
                     gammas: torch.Tensor, shot_list: Optional[torch.Tensor] = None,
                     list_count: Optional[torch.Tensor] = None, post_stride: int = 0) -> None:
        """propose() into caller-owned device buffers (no reshaping, no allocation); with
        ``shot_list`` / ``list_count`` (device int32) only those shots' rows are written.  ``post``
        is a tensor or a device address; row b starts ``post_stride`` floats after row b-1."""
        pp = ct.c_void_p(post) if isinstance(post, int) else _ptr(post)
        nat.check(nat.lib().rbp_net_propose(self._h, B, _ptr(syn), pp, int(post_stride), float(lo), float(hi),
                                            _ptr(shot_list), _ptr(list_count), _ptr(gammas), None, self._stream()),
                  "rbp_net_propose")

    def train_step(self, syn, post, target, cfg: TrainConfig, lr: float, loss_out: Optional[torch.Tensor] = None,
                   grads_out: Optional[torch.Tensor] = None) -> None:
        syn, post = self._inputs(syn, post)
        target = target.to(device=self.device, dtype=torch.uint8).contiguous()
        hp = nat.RbpNetHparams(lr=lr, beta1=cfg.beta1, beta2=cfg.beta2, eps=cfg.eps, weight_decay=cfg.weight_decay,
                               w_neg=cfg.w_neg)
        nat.check(nat.lib().rbp_net_train_step(self._h, syn.shape[0], _ptr(syn), _ptr(post), _ptr(target),
                                               ct.byref(hp), _ptr(loss_out), _ptr(grads_out), self._stream()),
                  "rbp_net_train_step")

    def save(self, path, meta: Optional[dict] = None) -> None:
        np.savez(path, params=self.params().cpu().numpy(), meta=json.dumps(meta or {}))


# ---------------------------------------------------------------------------- data generation


class ShotSampler:
    """Seeded shots on the device: e ~ Bernoulli(priors), s = H e mod 2."""

    def __init__(self, H_csr, priors, device, seed: int):
        self.device = torch.device(device)
        Hc = H_csr.tocsr()
        self.C, self.V = Hc.shape
        self.HT = torch.from_numpy(Hc.toarray().T.astype(np.float32)).to(self.device)  # [V, C]
        self.p = torch.from_numpy(np.asarray(priors, np.float32)).to(self.device)
        self.gen = torch.Generator(device=self.device)
        self.gen.manual_seed(seed)

    def sample(self, B: int):
        e = (torch.rand(B, self.V, generator=self.gen, device=self.device) < self.p).to(torch.uint8)
        s = torch.remainder(e.float() @ self.HT, 2).to(torch.uint8)
        return e, s


def make_tuples(decoder: RelayBPDecoder, syn: torch.Tensor, err: torch.Tensor):
    """(posterior after the pre-iterations, target [hard == e]) for each shot."""
    pre = decoder.decode_phases(syn, skip_relay_legs=True, return_last_posterior=True)
    post = pre["last_posterior"].float()
    target = ((post <= 0).to(torch.uint8) == err).to(torch.uint8)
    return post, target


def train(decoder: RelayBPDecoder, H_csr, priors, cfg: TrainConfig, net: Optional[ProposalNet] = None,
          log=print) -> tuple[ProposalNet, list]:
    """Train on cfg.tuples decoder-generated tuples; returns the network and the loss log."""
    net = net or ProposalNet(decoder, init_params(cfg.init_seed))
    sampler = ShotSampler(H_csr, priors, net.device, cfg.seed)
    steps = max(1, cfg.tuples // cfg.batch)
    loss = torch.zeros(1, device=net.device)
    hist, acc, t0 = [], torch.zeros(1, device=net.device), time.time()
    for step in range(steps):
        err, syn = sampler.sample(cfg.batch)
        post, target = make_tuples(decoder, syn, err)
        lr = cfg.lr_final + 0.5 * (cfg.lr - cfg.lr_final) * (1 + np.cos(np.pi * step / steps))
        net.train_step(syn, post, target, cfg, lr, loss_out=loss)
        acc += loss
        if (step + 1) % cfg.log_every == 0 or step + 1 == steps:
            k = (step % cfg.log_every) + 1
            mean = float(acc) / k
            acc.zero_()
            hist.append({"step": step + 1, "tuples": (step + 1) * cfg.batch, "loss": mean,
                         "seconds": time.time() - t0})
            log(json.dumps(hist[-1]))
    return net, hist


# ---------------------------------------------------------------------------- learned decode


class LearnedRelayBPDecoder:
    """Relay-BP with learned strengths for the first relay legs.

    ``decode(syndromes)`` runs three launches on the current stream: the
    pre-iterations (saving each shot's state and posterior), the network's
    tensor-core inference, and the relay legs resumed from the saved state with
    the proposed strengths on legs 0..learned_legs-1 and the seeded table after.
    The relay legs take the shots the pre-iterations left unconverged first.
    Outputs have the same keys as ``RelayBPDecoder.decode``.

    With ``gate=True`` the network is evaluated only for those unconverged
    shots (chosen on the device, no host round trip); a shot the
    pre-iterations solved keeps its posterior with the interval's top strength
    ``hi`` on the learned legs.  ``fused=True`` (gated only) lets a solved shot
    run on into its relay legs inside the first launch and resumes only the
    unconverged shots afterwards; same results, but those shots' legs then run
    after the bulk instead of beside it, which measured slower (17.0 vs 16.0 ms
    for 65,536 shots of the [[144,12,12]] phenomenological code, one B200).

    ``network=False`` (gated only) is the ablation without the network: solved
    shots still take ``hi`` on the learned legs, unconverged shots run the
    seeded legs, and the network launch is skipped.  It separates what the
    gate rule contributes from what the network contributes.

    With ``graph=True`` (default) the launches and the small device ops between
    them are captured once per batch size as a CUDA graph; a call then copies
    the syndromes into the captured input buffer and replays the graph.  Calls
    that pass ``events`` run eagerly.  Not for concurrent use from several
    streams: the buffers and graphs belong to the decoder object.

    ``decode_stream(batches)`` decodes a sequence of host batches with the
    host/device copies overlapped with the decodes (two sets of buffers and
    graphs, a copy stream).
    """

    def __init__(self, decoder: RelayBPDecoder, net: ProposalNet, learned_legs: int = 4, gate: bool = False,
                 fused: bool = False, graph: bool = True, network: bool = True):
        if decoder.algo != "relay":
            raise ValueError("learned legs need algo='relay'")
        if decoder.num_gpus != 1:
            raise ValueError("the learned decode runs on one GPU")
        self.dec, self.net = decoder, net
        self.learned_legs = int(min(learned_legs, decoder.num_sets))
        self.lo, self.hi = (float(x) for x in decoder.gamma_dist_interval)
        self.gate = bool(gate)
        self.network = bool(network)
        if not self.network and not self.gate:
            raise ValueError("network=False is the gate-only ablation: it needs gate=True")
        self.fused = bool(fused)
        self.graph = bool(graph)
        self._graphs: Dict[tuple, tuple] = {}  # (B, slot) -> (graph, static input, buffers)
        self._bufs: Dict[tuple, dict] = {}     # (B, slot) -> buffers
        self._copy_stream: Optional[torch.cuda.Stream] = None

    def _buffers(self, B: int, slot: int = 0) -> dict:
        b = self._bufs.get((B, slot))
        if b is None:
            if any(k[0] != B for k in self._bufs):
                self._bufs, self._graphs = {}, {}  # keep one batch size; graphs refer to their buffers
            d, dev = self.dec, self.net.device
            b = {
                "state": d.new_state(B),
                "gammas": torch.empty(B, d.V, dtype=torch.float32, device=dev),
                "found": torch.empty(B, dtype=torch.int32, device=dev),
                "iters": torch.empty(B, dtype=torch.int32, device=dev),
                "wfix": torch.empty(B, dtype=torch.int64, device=dev),
                "errors": torch.empty(B, d.V, dtype=torch.uint8, device=dev),
                "count": torch.empty(1, dtype=torch.int32, device=dev),
            }
            self._bufs[(B, slot)] = b
        return b

    def _graph_entry(self, syn: torch.Tensor, slot: int = 0) -> tuple:
        """(graph, static input, buffers) of this batch size and buffer set; captured on first
        use from an eager warm-up decode of ``syn``."""
        B = int(syn.shape[0])
        shapes = (self.dec._launch, self.dec._pre_launch)  # a graph keeps the kernel shapes it captured
        entry = self._graphs.get((B, slot))
        if entry is not None and entry[3] != shapes:
            entry = None
        if entry is None:
            static = torch.empty(B, self.dec.C, dtype=torch.uint8, device=self.net.device)
            static.copy_(syn)
            self.decode_into(static, slot=slot)  # eager warm-up: buffers, kernel attributes, allocator pool
            torch.cuda.synchronize(self.net.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                bf = self.decode_into(static, slot=slot)
            entry = (g, static, bf, shapes)
            self._graphs[(B, slot)] = entry
        return entry

    def _replay(self, syn: torch.Tensor) -> dict:
        """Copy the syndromes (host or device) into the captured input buffer and replay."""
        g, static, bf, _ = self._graph_entry(syn)
        static.copy_(syn, non_blocking=True)
        g.replay()
        return bf

    def decode_into(self, syn: torch.Tensor, events=None, slot: int = 0) -> dict:
        """Launch the three phases into the persistent buffers of this batch size (no host sync).
        ``events``: four CUDA events recorded before the pre-iterations, after them, after the
        network (with its shot selection) and after the relay legs."""
        d = self.dec
        B = int(syn.shape[0])
        bf = self._buffers(B, slot)
        gid = d.device_ids[0]
        stream = torch.cuda.current_stream(self.net.device).cuda_stream
        gamma0 = float(np.float32(d.gamma0))
        if self.gate and self.fused:
            return self._decode_gated(syn, B, bf, gid, stream, gamma0, events)
        if events is not None:
            events[0].record()
        pre_in = nat.RbpBatch(syndromes=_ptr(syn), gamma0=gamma0, pre_iter=d.pre_iter, skip_relay_legs=1,
                              suspend_state=_ptr(bf["state"]), parity_first=d.parity_first)
        pre_out = nat.RbpOutputs(found_count=_ptr(bf["found"]), iterations=_ptr(bf["iters"]))
        d._native[gid].decode(B, pre_in, pre_out, stream)
        if events is not None:
            events[1].record()
        unsolved = bf["found"] == 0
        order = torch.argsort((~unsolved).to(torch.uint8), stable=True).to(torch.int32)  # unconverged first
        post = bf["state"].data_ptr() + self._post_offset()  # posteriors, read from the saved states
        stride = bf["state"].shape[1] // 4
        if self.gate:
            # solved shots take the constant hi in the kernel; only unsolved rows are written
            if self.network:
                bf["count"].copy_(unsolved.sum().to(torch.int32).view(1))
                self.net.propose_into(B, syn, post, self.lo, self.hi, bf["gammas"], order, bf["count"],
                                      post_stride=stride)
        else:
            self.net.propose_into(B, syn, post, self.lo, self.hi, bf["gammas"], post_stride=stride)
        legs_in = nat.RbpBatch(syndromes=_ptr(syn), gamma0=gamma0, pre_iter=d.pre_iter,
                               gamma_legs_shot=_ptr(bf["gammas"] if self.network else None),
                               n_shot_legs=self.learned_legs if self.network else 0, shot_leg_rows=1,
                               resume_state=_ptr(bf["state"]), legs_begin=0, shot_order=_ptr(order),
                               solved_gamma=float(np.float32(self.hi)),
                               solved_legs=self.learned_legs if self.gate else 0, parity_first=d.parity_first)
        legs_out = nat.RbpOutputs(errors=_ptr(bf["errors"]), weight_fixed=_ptr(bf["wfix"]),
                                  found_count=_ptr(bf["found"]), iterations=_ptr(bf["iters"]))
        if events is not None:
            events[2].record()
        d._native[gid].decode(B, legs_in, legs_out, stream)
        if events is not None:
            events[3].record()
        return bf

    def _decode_gated(self, syn, B, bf, gid, stream, gamma0, events):
        """gate=True in three launches: (1) every shot's pre-iterations, after which a solved shot
        goes on through its relay legs with the top strength on the learned legs, and an unsolved
        shot saves its state and stops; (2) the network for the unsolved shots, reading their
        posteriors from the saved states; (3) their relay legs, resumed with the proposed
        strengths.  Identical results to the ungated order of work with strength hi on the solved
        shots' learned legs."""
        d = self.dec
        if events is not None:
            events[0].record()
        first_in = nat.RbpBatch(syndromes=_ptr(syn), gamma0=gamma0, pre_iter=d.pre_iter,
                                suspend_state=_ptr(bf["state"]), suspend_unsolved=1,
                                solved_gamma=float(np.float32(self.hi)), solved_legs=self.learned_legs)
        outs = nat.RbpOutputs(errors=_ptr(bf["errors"]), weight_fixed=_ptr(bf["wfix"]),
                              found_count=_ptr(bf["found"]), iterations=_ptr(bf["iters"]))
        d._native[gid].decode(B, first_in, outs, stream)
        if events is not None:
            events[1].record()
        unsolved = bf["found"] == 0
        order = torch.argsort((~unsolved).to(torch.uint8), stable=True).to(torch.int32)
        bf["count"].copy_(unsolved.sum().to(torch.int32).view(1))
        stride = bf["state"].shape[1]
        if self.network:
            self.net.propose_into(B, syn, bf["state"].data_ptr() + self._post_offset(), self.lo, self.hi,
                                  bf["gammas"], order, bf["count"], post_stride=stride // 4)
        if events is not None:
            events[2].record()
        legs_in = nat.RbpBatch(syndromes=_ptr(syn), gamma0=gamma0, pre_iter=d.pre_iter,
                               gamma_legs_shot=_ptr(bf["gammas"] if self.network else None),
                               n_shot_legs=self.learned_legs if self.network else 0, shot_leg_rows=1,
                               resume_state=_ptr(bf["state"]), legs_begin=0, shot_order=_ptr(order),
                               queue_len=_ptr(bf["count"]))
        d._native[gid].decode(B, legs_in, outs, stream)
        if events is not None:
            events[3].record()
        return bf

    def _post_offset(self) -> int:
        off = ct.c_int64()
        nat.check(nat.lib().rbp_state_posterior_offset(self.dec._native[self.dec.device_ids[0]]._dec,
                                                       ct.byref(off)), "rbp_state_posterior_offset")
        return int(off.value)

    def decode(self, syndromes: torch.Tensor, events=None) -> Dict[str, torch.Tensor]:
        d = self.dec
        if not isinstance(syndromes, torch.Tensor):
            syndromes = torch.as_tensor(np.asarray(syndromes))
        if syndromes.ndim != 2 or syndromes.shape[1] != d.C:
            raise ValueError(f"syndromes must be [B, {d.C}]")
        if syndromes.shape[0] == 0:
            return d.decode(syndromes)
        if self.graph and events is None:
            bf = self._replay(syndromes)  # host syndromes are copied straight into the graph's input
        else:
            bf = self.decode_into(syndromes.to(device=self.net.device, dtype=torch.uint8).contiguous(), events)
        wfix, found = bf["wfix"].clone(), bf["found"].clone()
        has = wfix != torch.iinfo(torch.int64).max
        weights = torch.where(has, wfix.to(torch.float64) * (2.0 ** -32),
                              torch.full_like(wfix, 0, dtype=torch.float64) + float("inf")).to(torch.float32)
        return {
            "errors": bf["errors"].clone(),
            "weights": weights,
            "valid_mask": found >= d.stop_nconv,
            "iterations": bf["iters"].clone(),
            "found_count": found,
            "unconverged_indices": torch.nonzero(found < d.stop_nconv).flatten().to(torch.int32),
            "weight_fixed": wfix,
        }

    STREAM_KEYS = (("errors", "errors", torch.uint8), ("weight_fixed", "wfix", torch.int64),
                   ("found_count", "found", torch.int32), ("iterations", "iters", torch.int32))

    def decode_stream(self, batches: Sequence[torch.Tensor],
                      out: Optional[Sequence[Dict[str, torch.Tensor]]] = None) -> List[Dict[str, torch.Tensor]]:
        """Decode a sequence of host syndrome batches, all [B, C] uint8 on the CPU (pinned for
        the copies to overlap), with the transfers hidden behind the decodes.  Two sets of
        device buffers and captured graphs alternate: while batch i decodes on the current
        stream, a copy stream brings batch i+1's syndromes in and batch i-1's results out.

        ``out[i]`` (CPU tensors, pinned for overlap; allocated pinned when ``out`` is None)
        receives batch i's ``errors`` [B, V] uint8, ``weight_fixed`` [B] int64, ``found_count``
        and ``iterations`` [B] int32 -- the same values ``decode`` returns for that batch.  Entries
        of ``out`` may repeat (a ring of host buffers); each is written in batch order.  Returns
        after every copy has finished."""
        n = len(batches)
        if n == 0:
            return []
        d, dev = self.dec, self.net.device
        B = int(batches[0].shape[0])
        for x in batches:
            if x.device.type != "cpu" or x.dtype != torch.uint8 or tuple(x.shape) != (B, d.C):
                raise ValueError(f"decode_stream takes CPU uint8 batches of shape [{B}, {d.C}]")
        if B == 0:
            raise ValueError("decode_stream needs non-empty batches")
        if out is None:
            out = [{k: torch.empty((B, d.V) if k == "errors" else (B,), dtype=t).pin_memory()
                    for k, _, t in self.STREAM_KEYS} for _ in range(n)]
        if len(out) != n:
            raise ValueError("out must hold one entry per batch")
        entries = [self._graph_entry(batches[0], slot) for slot in range(min(2, n))]
        compute = torch.cuda.current_stream(dev)
        if self._copy_stream is None:
            self._copy_stream = torch.cuda.Stream(dev)
        copy = self._copy_stream
        start = torch.cuda.Event()
        start.record(compute)
        copy.wait_event(start)
        h2d: List[Optional[torch.cuda.Event]] = [None] * n

        def bring_in(i: int) -> None:
            # on the copy stream after batch i-2's results left the same buffers
            with torch.cuda.stream(copy):
                entries[i % 2][1].copy_(batches[i], non_blocking=True)
                h2d[i] = torch.cuda.Event()
                h2d[i].record(copy)

        bring_in(0)
        for i in range(n):
            g, _, bf, _ = entries[i % 2]
            compute.wait_event(h2d[i])
            g.replay()
            decoded = torch.cuda.Event()
            decoded.record(compute)
            if i + 1 < n:
                bring_in(i + 1)
            with torch.cuda.stream(copy):
                copy.wait_event(decoded)
                for key, buf, _ in self.STREAM_KEYS:
                    out[i][key].copy_(bf[buf], non_blocking=True)
        finished = torch.cuda.Event()
        finished.record(copy)
        compute.wait_event(finished)  # work queued after this call sees the results in place
        finished.synchronize()
        return list(out)


def default_weights_path(workload: str = "bb144_phen", p: float = 0.003) -> Path:
    return DATA_DIR / f"proposal_{workload}_p{str(p).replace('.', '')}.npz"


# ---------------------------------------------------------------------------- evaluation and CLI


def _timed(fn):
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1)


def constant_params(logit: float = 20.0) -> np.ndarray:
    """Parameters of a network whose every output is sigmoid(logit): the constant-strength ablation."""
    theta = np.zeros(param_count(), np.float32)
    theta[-1] = logit
    return theta


def evaluate(workload, net: ProposalNet, decoder: RelayBPDecoder, shots: int, seed: int, chunk: int = 262144,
             learned_legs: int = 4,
             variants=("plain", "learned", "learned_gated", "gate_no_network", "constant_hi")) -> dict:
    """Decode the same fresh seeded shots with each variant: logical error rate (Wilson 95% interval),
    mean iterations and decode time (device time, syndromes resident, one call per chunk).

    plain          the decoder alone (seeded legs)
    learned        network strengths on legs 0..learned_legs-1 for every shot
    learned_gated  network strengths for the shots the pre-iterations left unconverged, the top
                   strength hi for the others
    gate_no_network  the gate rule alone: hi on the learned legs for the shots the pre-iterations
                   solved, the seeded legs for the others (no network): separates the rule from
                   the network
    constant_hi    strength hi (a network with constant output) for every shot: the ablation
    """
    from .experiments import wilson

    const_net = ProposalNet(decoder, constant_params())
    runners = {
        "plain": decoder.decode,
        "learned": LearnedRelayBPDecoder(decoder, net, learned_legs).decode,
        "learned_gated": LearnedRelayBPDecoder(decoder, net, learned_legs, gate=True).decode,
        "gate_no_network": LearnedRelayBPDecoder(decoder, net, learned_legs, gate=True, network=False).decode,
        "constant_hi": LearnedRelayBPDecoder(decoder, const_net, learned_legs).decode,
    }
    rows = {v: {"fails": 0, "unconv": 0, "iters": 0, "ms": 0.0} for v in variants}
    done, k = 0, 0
    gamma_stats = None
    while done < shots:
        n = min(chunk, shots - done)
        err, syn = workload.sample(n, seed=seed + k)
        syn_d = torch.from_numpy(syn).to(net.device)
        if k == 0:
            for v in variants:
                runners[v](syn_d)  # warm-up at this size
            pre = decoder.decode_phases(syn_d, skip_relay_legs=True, return_last_posterior=True)
            g = net.propose(syn_d, pre["last_posterior"], *decoder.gamma_dist_interval)
            solved = pre["found_count"] > 0
            gamma_stats = {"mean_gamma_solved": float(g[solved].mean()),
                           "frac_below_0p6_solved": float((g[solved] < 0.6).float().mean()),
                           "mean_gamma_unsolved": float(g[~solved].mean()) if bool((~solved).any()) else None,
                           "frac_below_0p6_unsolved": float((g[~solved] < 0.6).float().mean())
                           if bool((~solved).any()) else None,
                           "unsolved_after_pre_iterations": int((~solved).sum())}
        for v in variants:
            out, ms = _timed(lambda: runners[v](syn_d))
            o = {kk: x.cpu().numpy() for kk, x in out.items() if isinstance(x, torch.Tensor)}
            conv = o["found_count"] > 0
            f = workload.logical_failures(err, o["errors"], conv)
            r = rows[v]
            r["fails"] += int(f.sum())
            r["unconv"] += int((~conv).sum())
            r["iters"] += int(o["iterations"].astype(np.int64).sum())
            r["ms"] += ms
        done += n
        k += 1
    res = {"shots": shots, "seed": seed, "learned_legs": learned_legs, "chunk": chunk,
           "network_outputs_first_chunk": gamma_stats}
    for v, r in rows.items():
        lo, hi = wilson(r["fails"], shots)
        res[v] = {"ler": r["fails"] / shots, "ler_ci95": [lo, hi], "failures": r["fails"],
                  "unconverged": r["unconv"], "mean_iterations": r["iters"] / shots,
                  "decode_ms": r["ms"], "shots_per_s": shots / (r["ms"] * 1e-3)}
    if "plain" in rows:
        pl = res["plain"]
        for v in variants:
            if v == "plain":
                continue
            res[v]["speedup_vs_plain"] = res[v]["shots_per_s"] / pl["shots_per_s"]
            res[v]["iteration_ratio_vs_plain"] = pl["mean_iterations"] / res[v]["mean_iterations"]
            ci = res[v]["ler_ci95"]
            res[v]["ler_within_plain_ci"] = bool(ci[0] <= pl["ler_ci95"][1] and pl["ler_ci95"][0] <= ci[1])
    return res


def main(argv=None):
    import argparse

    from . import codes

    ap = argparse.ArgumentParser(prog="python -m pelagos_b200.proposal")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="train on decoder-generated tuples and save the weights")
    t.add_argument("--workload", default="bb144_phen")
    t.add_argument("--p", type=float, default=0.003)
    t.add_argument("--tuples", type=int, default=1 << 22)
    t.add_argument("--batch", type=int, default=1024)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--w-neg", type=float, default=20.0)
    t.add_argument("--seed", type=int, default=2024)
    t.add_argument("--out", default=None)
    e = sub.add_parser("eval", help="plain vs learned decode on fresh seeded shots")
    e.add_argument("--workload", default="bb144_phen")
    e.add_argument("--p", type=float, default=0.003)
    e.add_argument("--weights", default=None)
    e.add_argument("--shots", type=int, default=1 << 20)
    e.add_argument("--seed", type=int, default=900001)
    e.add_argument("--out", default=None)
    c = sub.add_parser("propose-case", help="a small inference case: pre-iterations, then the network 3 times")
    c.add_argument("--workload", default="bb144_phen")
    c.add_argument("--p", type=float, default=0.003)
    c.add_argument("--shots", type=int, default=4096)
    a = ap.parse_args(argv)
    w = codes.workload(a.workload, p=a.p)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    if a.cmd == "propose-case":
        net = ProposalNet(dec, load_params(default_weights_path(a.workload, a.p))[0])
        syn = torch.from_numpy(w.sample(a.shots, seed=1)[1]).to(net.device)
        pre = dec.decode_phases(syn, skip_relay_legs=True, return_last_posterior=True)
        for _ in range(3):
            g = net.propose(syn, pre["last_posterior"], *dec.gamma_dist_interval)
        torch.cuda.synchronize()
        print(json.dumps({"shots": a.shots, "mean_gamma": float(g.mean())}))
        return
    if a.cmd == "train":
        cfg = TrainConfig(tuples=a.tuples, batch=a.batch, lr=a.lr, w_neg=a.w_neg, seed=a.seed)
        net, hist = train(dec, w.H, w.priors, cfg)
        out = a.out or str(default_weights_path(a.workload, a.p))
        Path(out).parent.mkdir(parents=True, exist_ok=True)
        net.save(out, meta={"workload": a.workload, "p": a.p, "train": asdict(cfg), "log": hist[-8:],
                            "decoder": RELAY})
        print(json.dumps({"saved": out, "final_loss": hist[-1]["loss"], "seconds": hist[-1]["seconds"]}))
    else:
        params, meta = load_params(a.weights or default_weights_path(a.workload, a.p))
        net = ProposalNet(dec, params)
        res = evaluate(w, net, dec, a.shots, a.seed)
        res["weights_meta"] = {k: meta.get(k) for k in ("workload", "p", "train")}
        print(json.dumps(res, indent=1))
        if a.out:
            Path(a.out).write_text(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
