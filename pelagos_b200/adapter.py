"""relay_bp-style adapter over the B200 decoder: ``RelayDecoder`` and
``ObservableDecoderRunner``, the entry points the reference's benchmark and
tutorials use (src/pelagos/adapter.py:86-858).

``RelayDecoder`` maps the three configuration dicts of the reference
(``msl_config``, ``relay_config``, ``backend_config``) onto
``pelagos_b200.RelayBPDecoder`` and offers the same decode methods and
``DecodeResult`` records.  ``ObservableDecoderRunner`` decodes batches of error
patterns and reports the logical observables; unlike the reference, which forms
s = H e and O e / O e_hat on the host with scipy (adapter.py:545-560, 601-613,
679), it forms both on the GPU (``rbp_gf2_matvec``) and copies the results to
the host once per batch.

Extensions: ``backend_config["proposal"]`` (a weights file, or ``"default"``
for the packaged network of the decoder's workload) makes the adapter decode
with learned relay legs (``LearnedRelayBPDecoder``, gated);
``data_type="bfloat16"`` is accepted.  ``execution="process"`` (the
reference's process-per-GPU backend) and layered scheduling are not provided.
"""

from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np
import scipy.sparse as sp
import torch

from . import _native as nat
from .decoder import RelayBPDecoder, _ptr

_DTYPE_ALIASES = {"float": "float32", "half": "float16", "double": "float64", "fp16": "float16",
                  "fp32": "float32", "fp64": "float64", "bf16": "bfloat16"}


@dataclass
class DecodeResult:
    """One shot's result, shaped like the relay_bp ``DecodeResult`` / ``ObservableDecodeResult``
    (adapter.py:41-83): ``decoding``, ``success`` and ``iterations`` are the relay_bp fields; the
    rest are filled where the calling method knows them."""

    decoding: np.ndarray
    success: bool
    iterations: int
    decoding_quality: float = float("inf")
    unconverged_no_error: Optional[bool] = None
    unconverged_logical_error: Optional[bool] = None
    better_decoding_quality_error: Optional[bool] = None
    worse_decoding_quality_error: Optional[bool] = None
    converged: bool = False
    error_detected: bool = False
    observables: np.ndarray = None  # type: ignore[assignment]
    unconverged_indices: Optional[np.ndarray] = None
    found_count: Optional[int] = None


def _as_u8_tensor(x) -> torch.Tensor:
    if isinstance(x, np.ndarray):
        return torch.from_numpy(np.ascontiguousarray(x.astype(np.uint8, copy=False)))
    return x.to(dtype=torch.uint8)


class _DeviceCSR:
    """A sparse 0/1 matrix on the device for rbp_gf2_matvec."""

    def __init__(self, A, device):
        A = sp.csr_matrix(A)
        A.sort_indices()
        self.R, self.N = A.shape
        self.row_ptr = torch.from_numpy(A.indptr.astype(np.int32)).to(device)
        self.cols = torch.from_numpy(A.indices.astype(np.int32)).to(device)

    def apply(self, x: torch.Tensor) -> torch.Tensor:
        """[B, N] uint8 device rows -> [B, R] uint8 parities."""
        x = x.to(dtype=torch.uint8).contiguous()
        B = int(x.shape[0])
        out = torch.empty(B, self.R, dtype=torch.uint8, device=x.device)
        nat.check(nat.lib().rbp_gf2_matvec(_ptr(x), B, self.N, _ptr(self.row_ptr), _ptr(self.cols), self.R,
                                           _ptr(out), ct.c_void_p(torch.cuda.current_stream(x.device).cuda_stream)),
                  "rbp_gf2_matvec")
        return out


class RelayDecoder:
    """Relay-BP decoder behind the relay_bp-style interface (adapter.py:86-512)."""

    def __init__(self, check_matrix, *, msl_config: Optional[dict] = None, relay_config: Optional[dict] = None,
                 data_type: Optional[str] = None, backend_config: Optional[dict] = None, **kwargs):
        if msl_config is None or relay_config is None:
            raise ValueError("msl_config and relay_config must be provided to RelayDecoder")
        msl, relay, backend = dict(msl_config), dict(relay_config), dict(backend_config or {})
        error_priors = msl.get("error_priors")
        if error_priors is None:
            raise ValueError("msl_config must contain 'error_priors'")
        dt = backend.get("data_type", data_type)
        dt = _DTYPE_ALIASES.get(dt, dt)
        if dt not in ("float16", "float32", "float64", "bfloat16"):
            raise ValueError(f"Unsupported data_type: {dt!r}")
        self.data_type = dt
        if backend.get("execution", "thread") != "thread":
            raise NotImplementedError("execution='process' (a worker process per GPU) is not provided; "
                                      "device=[...] runs one replica per GPU in this process")
        device = backend.get("device", (0,))
        device = list(device) if isinstance(device, tuple) else ([device] if isinstance(device, int) else device)
        self.stop_nconv = int(relay.get("stop_nconv", 1))
        num_sets = int(relay.get("num_sets", 300))
        interval = (0.0, 0.0) if num_sets == 0 else tuple(relay.get("gamma_dist_interval", (-0.24, 0.66)))
        self.H_csr = sp.csr_matrix(check_matrix)
        self.N = int(self.H_csr.shape[1])
        seed = relay.get("seed", 0)
        self._dec = RelayBPDecoder(
            self.H_csr, error_priors=error_priors,
            pre_iter=int(relay.get("pre_iter", 80)), num_sets=num_sets,
            set_max_iter=int(relay.get("set_max_iter", 60)), gamma0=float(msl.get("gamma0", 0.1)),
            gamma_dist_interval=interval, stop_nconv=self.stop_nconv,
            normalized_min_sum_alpha=msl.get("alpha", None), offset_min_sum_beta=msl.get("beta", None),
            data_type=dt, device=device, seed=int(seed) if seed is not None else 0,
            gamma_draw=str(relay.get("gamma_draw", "broadcast")),
            bitpack_output=bool(backend.get("bitpack_output", False)), algo=backend.get("algo", "relay"),
            perf=backend.get("perf", "throughput"),
            alpha_iteration_scaling_factor=float(msl.get("alpha_iteration_scaling_factor", 1.0)),
            explicit_gammas=relay.get("explicit_gammas", None),
            gamma_dist_interval_by_error=relay.get("gamma_dist_interval_by_error", None),
            fast_max_unconverged_pct=backend.get("fast_max_unconverged_pct", None),
            scheduling=backend.get("scheduling", "flood-fill"),
            unconverged_correction=str(relay.get("unconverged_correction", "first_leg")),
        )
        self._process_execution = False
        self._learned = None
        proposal = backend.get("proposal")
        if proposal is not None:
            self._learned = self._make_learned(proposal, backend)

    def _make_learned(self, proposal, backend):
        from .proposal import LearnedRelayBPDecoder, ProposalNet, load_params

        if self._dec.bitpack_output:
            raise ValueError("the learned decode returns unpacked errors; use bitpack_output=False")
        if proposal == "default":
            from .proposal import default_weights_path

            proposal = default_weights_path()
        params, _ = load_params(proposal)
        return LearnedRelayBPDecoder(self._dec, ProposalNet(self._dec, params),
                                     learned_legs=int(backend.get("learned_legs", 4)),
                                     gate=bool(backend.get("gate", True)))

    # ------------------------------------------------------------------ housekeeping

    def close(self):
        """Nothing to release (no worker processes)."""

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _decode_inner(self, S_torch) -> Dict[str, torch.Tensor]:
        """The one place that decodes: the decoder's (or the learned decoder's) result dict."""
        if self._learned is not None:
            return self._learned.decode(S_torch)
        return self._dec.decode(S_torch)

    def log_prior_ratios(self) -> np.ndarray:
        """ln((1-p)/p) per column with non-finite entries zeroed (the quality weights)."""
        return np.asarray(self._dec.wj, dtype=np.float64)

    def override_llr_columns(self, cols, value: float):
        """Set the prior LLR of columns; returns a callable that restores them."""
        return self._dec.override_llr_columns(cols, value)

    # ------------------------------------------------------------------ decode methods

    def decode(self, syndrome):
        """One syndrome -> dict(bits, posterior_llr, converged, num_ensembles, iterations, selected_idx)."""
        s = _as_u8_tensor(syndrome).reshape(1, -1)
        out = self._decode_inner(s)
        res = {
            "bits": out["errors"][0].to(torch.int8),
            "posterior_llr": None,
            "converged": bool(int(out["found_count"][0]) > 0),
            "num_ensembles": 0,
            "iterations": int(out["iterations"][0]),
            "selected_idx": 0,
        }
        if "unconverged_indices" in out:
            res["unconverged_indices"] = out["unconverged_indices"].cpu().numpy()
        return res

    def decode_detailed(self, detectors) -> DecodeResult:
        r = self.decode(detectors)
        bits = r["bits"].cpu().numpy()
        ok = bool(r["converged"])
        return DecodeResult(decoding=bits, success=ok, iterations=int(r["iterations"]), converged=ok,
                            error_detected=not ok, observables=bits,
                            unconverged_indices=r.get("unconverged_indices"))

    def decode_batch(self, detectors, return_iterations: bool = False):
        """[B, C] -> int8 errors [B, V] (plus unconverged indices when fast_max_unconverged_pct is set,
        plus per-shot iterations when asked)."""
        out = self._decode_inner(_as_u8_tensor(detectors))
        res = [out["errors"].to(torch.int8).cpu().numpy()]
        if self._dec.fast_max_unconverged_pct is not None and "unconverged_indices" in out:
            res.append(out["unconverged_indices"].cpu().numpy())
        if return_iterations:
            res.append(out["iterations"].to(torch.int32).cpu().numpy())
        return res[0] if len(res) == 1 else tuple(res)

    def decode_batch_with_prior_tensors(self, detectors: torch.Tensor, prior_llr: torch.Tensor, *,
                                        return_iterations: bool = False):
        """Per-shot [B, V] prior LLRs in, (errors, last posterior[, iterations]) out, on the device."""
        out = self._dec.decode(detectors, return_last_posterior=True, prior_llr=prior_llr)
        if return_iterations:
            return out["errors"], out["last_posterior"], out["iterations"]
        return out["errors"], out["last_posterior"]

    def _records(self, out, B, with_quality: bool) -> List[DecodeResult]:
        bits = out["errors"].to(torch.int8).cpu().numpy()
        iters = out["iterations"].cpu().numpy()
        found = out["found_count"].cpu().numpy()
        unc_t = out.get("unconverged_indices")
        if with_quality:  # from_syndromes: the indices whenever there are any
            unc = unc_t.cpu().numpy() if (unc_t is not None and unc_t.numel() > 0) else None
        else:             # detailed_batch: only in the early-exit mode
            unc = unc_t.cpu().numpy() if (unc_t is not None and self._dec.fast_max_unconverged_pct is not None) \
                else None
        wj = self.log_prior_ratios() if with_quality else None
        recs = []
        for i in range(B):
            ok = bool(found[i] > 0)
            dq = float(np.dot(bits[i].astype(np.float64), wj)) if (with_quality and ok) else float("inf")
            recs.append(DecodeResult(decoding=bits[i], success=ok, iterations=int(iters[i]), decoding_quality=dq,
                                     converged=ok, error_detected=not ok, observables=bits[i],
                                     unconverged_indices=unc, found_count=int(found[i])))
        return recs

    def decode_detailed_batch(self, detectors) -> List[DecodeResult]:
        S = _as_u8_tensor(detectors)
        return self._records(self._decode_inner(S), int(S.shape[0]), with_quality=False)

    def decode_detailed_batch_from_syndromes(self, detectors) -> List[DecodeResult]:
        """The entry point higher-level decoders use: records with decoding_quality = e_hat . wj."""
        S = _as_u8_tensor(detectors)
        return self._records(self._decode_inner(S), int(S.shape[0]), with_quality=True)


# Aliases of the relay_bp class names the reference also exports.
RelayDecoderF32 = RelayDecoder
RelayDecoderF64 = RelayDecoder


class ObservableDecoderRunner:
    """Decode batches of error patterns and report observables and logical errors (adapter.py:515-858)."""

    def __init__(self, decoder: RelayDecoder, observables_matrix, include_decode_result: bool = True, **kwargs):
        self.decoder = decoder
        self._obs = sp.csr_matrix(observables_matrix)
        self.O, self.N = self._obs.shape
        self.M = int(decoder.H_csr.shape[0])
        dev = torch.device(f"cuda:{decoder._dec.device_ids[0]}")
        self._device = dev
        self._H_dev = _DeviceCSR(decoder.H_csr, dev)
        self._O_dev = _DeviceCSR(self._obs, dev)

    def _mul_mod2(self, A_csr, x) -> np.ndarray:
        """Host A x mod 2 (kept for callers of the reference's helper)."""
        y = sp.csr_matrix(A_csr) @ np.asarray(x, dtype=np.int64)
        return (np.asarray(y) % 2).astype(np.uint8)

    def from_errors_decode_observables_detailed_batch(self, errors: np.ndarray,
                                                      parallel: bool = False) -> List[DecodeResult]:
        return self._process_gpu_results(self._decode_gpu_only(errors))

    def _decode_gpu_only(self, errors: np.ndarray) -> Dict[str, object]:
        """Syndromes and true observables on the GPU, then the decode; nothing copied back yet."""
        B, N = errors.shape
        if N != self.decoder.N:
            raise ValueError(f"N mismatch: errors has {N}, decoder has {self.decoder.N}")
        e_dev = torch.from_numpy(np.ascontiguousarray(errors.astype(np.uint8, copy=False))).to(self._device)
        S = self._H_dev.apply(e_dev)
        perm = self.decoder._dec.check_permutation
        if perm is not None:
            S = S[:, torch.as_tensor(perm, device=self._device, dtype=torch.long)].contiguous()
        out = self.decoder._decode_inner(S)
        return {"out": out, "true_obs_dev": self._O_dev.apply(e_dev), "errors": errors}

    def _process_gpu_results(self, gpu_result: Dict[str, object]) -> List[DecodeResult]:
        return self._process_gpu_results_batched([gpu_result], [gpu_result["errors"]], [None])[0]

    def _process_gpu_results_batched(self, chunk_gpu_results, chunk_errors_list, chunk_true_obs_list):
        """Records for several decoded batches: predicted observables on the GPU, one copy each."""
        results = []
        wj = self.decoder.log_prior_ratios()
        for r, errors, true_obs in zip(chunk_gpu_results, chunk_errors_list, chunk_true_obs_list):
            out = r["out"]
            e_hat = out["errors"].to(torch.uint8)
            pred_obs = self._O_dev.apply(e_hat).cpu().numpy()
            if true_obs is None:
                true_obs = r["true_obs_dev"].cpu().numpy() if "true_obs_dev" in r \
                    else self._mul_mod2(self._obs, errors.T).T
            bits = e_hat.cpu().numpy()
            iters = out["iterations"].cpu().numpy()
            found = out["found_count"].cpu().numpy()
            unc = None
            if self.decoder._dec.fast_max_unconverged_pct is not None and out.get("unconverged_indices") is not None:
                unc = out["unconverged_indices"].cpu().numpy()
            dec_q = (bits.astype(np.float64) * wj).sum(axis=1)
            true_q = (errors.astype(np.float64) * wj).sum(axis=1)
            recs = []
            for i in range(errors.shape[0]):
                det = bool((true_obs[i] != pred_obs[i]).any())
                ok = bool(found[i] > 0)
                dq = float(dec_q[i]) if ok else float("inf")
                better = dq < true_q[i]
                recs.append(DecodeResult(
                    decoding=bits[i], success=ok, iterations=int(iters[i]), decoding_quality=dq,
                    unconverged_no_error=bool(not det and not ok), unconverged_logical_error=bool(det and not ok),
                    better_decoding_quality_error=bool(ok and det and better),
                    worse_decoding_quality_error=bool(ok and det and not better),
                    converged=ok, error_detected=det, observables=pred_obs[i].astype(np.uint8),
                    unconverged_indices=unc))
            results.append(recs)
        return results
