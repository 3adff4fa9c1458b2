"""MixedDecoder: several codes' syndrome batches in one persistent launch.

Each RelayBPDecoder keeps its own graph, priors, gamma table and parameters.
MixedDecoder hands all of their batches to one launch of the mixed-code
kernel (rbp_mixed_* in include/relaybp.h): thread blocks take shots from a
per-code work queue with that code's group shape and move to another code
when their queue runs dry, so codes of very different size share the GPU
without a launch per code.  With ``graph=True`` the launch (queue reset +
persistent kernel) is captured once per combination of batch sizes as a CUDA
graph and replayed; inputs are copied into persistent device buffers first.

Per-shot results are identical to decoding each batch with its own decoder
(the same kernel body runs each shot).  Only plain syndromes are supported
(no per-shot priors, initial posteriors or gammas).
"""

from __future__ import annotations

import ctypes as ct
from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from . import _native as nat
from .decoder import RelayBPDecoder, _ptr


class MixedDecoder:
    def __init__(self, decoders: Sequence[RelayBPDecoder], graph: bool = True):
        if not decoders:
            raise ValueError("MixedDecoder needs at least one decoder")
        dev = decoders[0].device_ids[0]
        for d in decoders:
            if d.num_gpus != 1 or d.device_ids[0] != dev:
                raise ValueError("all decoders of a MixedDecoder must run on the same single GPU")
            if d.dtype_str != "float32":
                raise NotImplementedError("mixed launches use float32 messages")
            if d.bitpack_output:
                raise NotImplementedError("bitpack_output is not supported in mixed launches")
            if d.gamma_draw == "per_row" and d._explicit_gammas is None and d.num_sets > 0:
                raise NotImplementedError("gamma_draw='per_row' is not supported in mixed launches")
        self.decoders = list(decoders)
        self.device = dev
        self.use_graph = graph
        handles = (ct.c_void_p * len(decoders))(*[d._native[dev]._dec for d in decoders])
        self._m = ct.c_void_p()
        nat.check(nat.lib().rbp_mixed_create(handles, len(decoders), ct.byref(self._m)), "rbp_mixed_create")
        self._captured: Tuple[int, ...] | None = None
        self._bufs: List[Dict[str, torch.Tensor]] = []

    def launch_info(self) -> List[dict]:
        out = []
        for i in range(len(self.decoders)):
            g, n, t, b = ct.c_int32(), ct.c_int32(), ct.c_int32(), ct.c_int32()
            nat.check(nat.lib().rbp_mixed_query(self._m, i, ct.byref(g), ct.byref(n), ct.byref(t), ct.byref(b)),
                      "rbp_mixed_query")
            out.append({"group_threads": g.value, "groups_per_block": n.value, "block_threads": t.value,
                        "blocks": b.value})
        return out

    def configure(self, group_threads: Sequence[int]) -> None:
        """Set each code's group size in the launch (0 keeps a code's current size); the next
        decode re-captures its graph."""
        if len(group_threads) != len(self.decoders):
            raise ValueError(f"expected {len(self.decoders)} group sizes")
        arr = (ct.c_int32 * len(group_threads))(*[int(g) for g in group_threads])
        nat.check(nat.lib().rbp_mixed_configure(self._m, arr), "rbp_mixed_configure")
        self._captured = None

    def _alloc(self, sizes: Tuple[int, ...]):
        dev = f"cuda:{self.device}"
        self._bufs = []
        for d, B in zip(self.decoders, sizes):
            self._bufs.append({
                "syndromes": torch.zeros(B, d.C, dtype=torch.uint8, device=dev),
                "errors": torch.empty(B, d.V, dtype=torch.uint8, device=dev),
                "weight_fixed": torch.empty(B, dtype=torch.int64, device=dev),
                "found_count": torch.empty(B, dtype=torch.int32, device=dev),
                "iterations": torch.empty(B, dtype=torch.int32, device=dev),
            })

    def _structs(self, sizes):
        n = len(self.decoders)
        Bs = (ct.c_int64 * n)(*sizes)
        ins = (nat.RbpBatch * n)()
        outs = (nat.RbpOutputs * n)()
        for i, (d, buf) in enumerate(zip(self.decoders, self._bufs)):
            gamma0 = float(np.float32(d.gamma0)) if d.algo == "relay" else 0.0
            ins[i] = nat.RbpBatch(syndromes=_ptr(buf["syndromes"]), gamma0=gamma0, pre_iter=d.pre_iter,
                                  parity_first=d.parity_first)
            outs[i] = nat.RbpOutputs(errors=_ptr(buf["errors"]), weight_fixed=_ptr(buf["weight_fixed"]),
                                     found_count=_ptr(buf["found_count"]), iterations=_ptr(buf["iterations"]))
        return Bs, ins, outs

    def decode(self, syndromes: Sequence[torch.Tensor]) -> List[Dict[str, torch.Tensor]]:
        """Decode syndromes[i] ([B_i, C_i] uint8) with decoders[i]; one result dict per decoder."""
        if len(syndromes) != len(self.decoders):
            raise ValueError(f"expected {len(self.decoders)} syndrome batches")
        sizes = tuple(int(s.shape[0]) for s in syndromes)
        for d, s in zip(self.decoders, syndromes):
            if s.ndim != 2 or s.shape[1] != d.C:
                raise ValueError(f"Expected {d.C} syndrome bits, got shape {tuple(s.shape)}")
        stream = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            if self._captured != sizes or not self._bufs or not self.use_graph:
                if not self._bufs or tuple(b["syndromes"].shape[0] for b in self._bufs) != sizes:
                    self._alloc(sizes)
                    self._captured = None
            for buf, s in zip(self._bufs, syndromes):
                buf["syndromes"].copy_(s, non_blocking=True)
            Bs, ins, outs = self._structs(sizes)
            if self.use_graph:
                if self._captured != sizes:
                    torch.cuda.synchronize(self.device)
                    nat.check(nat.lib().rbp_mixed_capture(self._m, Bs, ins, outs), "rbp_mixed_capture")
                    self._captured = sizes
                nat.check(nat.lib().rbp_mixed_replay(self._m, ct.c_void_p(stream.cuda_stream)), "rbp_mixed_replay")
            else:
                nat.check(nat.lib().rbp_mixed_decode(self._m, Bs, ins, outs, ct.c_void_p(stream.cuda_stream)),
                          "rbp_mixed_decode")
            results = []
            for d, buf in zip(self.decoders, self._bufs):
                wfix = buf["weight_fixed"].clone()
                found = buf["found_count"].clone()
                has = wfix != torch.iinfo(torch.int64).max
                weights = torch.where(has, wfix.to(torch.float64) * (2.0 ** -32),
                                      torch.full_like(wfix, 0, dtype=torch.float64) + float("inf")).to(torch.float32)
                results.append({
                    "errors": buf["errors"].clone(),
                    "weights": weights,
                    "valid_mask": found >= d.stop_nconv,
                    "iterations": buf["iterations"].clone(),
                    "found_count": found,
                    "unconverged_indices": torch.nonzero(found < d.stop_nconv).flatten().to(torch.int32),
                    "weight_fixed": wfix,
                })
            return results

    def close(self):
        if getattr(self, "_m", None):
            nat.lib().rbp_mixed_destroy(self._m)
            self._m = ct.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass
