"""Monte-Carlo logical-error-rate estimation with every step on the GPU.

The reference's benchmark loop (pelagos_benchmark.py:1190-1197, 1462-1520,
1667-1669) samples errors and forms syndromes on the host, decodes on the GPU
and counts failures on the host.  Here one batch is:

1. seeded Bernoulli(priors) errors drawn on the device (torch's Philox
   generator, one generator per run, so a seed fixes the whole run);
2. syndromes s = H e with the library's GF(2) product kernel;
3. the decode (any decoder with ``decode(syndromes) -> dict``: the plain
   ``RelayBPDecoder``, ``LearnedRelayBPDecoder``, ...);
4. observables O e and O e_hat with the same kernel, and the failure count
   (an unconverged shot, or O (e + e_hat) != 0) reduced on the device.

Only a few integers per batch come back to the host.  ``run`` returns the
failure count, its Wilson 95 % interval, unconverged shots, mean iterations
and the decode throughput.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np
import scipy.sparse as sp
import torch

from .adapter import _DeviceCSR


def wilson(k: int, n: int, z: float = 1.959964) -> tuple[float, float]:
    if n == 0:
        return (0.0, 1.0)
    p = k / n
    d = 1 + z * z / n
    c = (p + z * z / (2 * n)) / d
    h = z * math.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return (max(0.0, c - h), min(1.0, c + h))


@dataclass
class MCResult:
    shots: int
    failures: int
    unconverged: int
    logical_flips: int
    mean_iterations: float
    decode_seconds: float
    ler: float = field(init=False)
    ler_ci95: tuple = field(init=False)

    def __post_init__(self):
        self.ler = self.failures / self.shots if self.shots else 0.0
        self.ler_ci95 = wilson(self.failures, self.shots)

    def as_dict(self) -> dict:
        return {"shots": self.shots, "failures": self.failures, "ler": self.ler, "ler_ci95": list(self.ler_ci95),
                "unconverged": self.unconverged, "logical_flips": self.logical_flips,
                "mean_iterations": self.mean_iterations, "decode_seconds": self.decode_seconds,
                "shots_per_s": self.shots / self.decode_seconds if self.decode_seconds else None}


class MonteCarlo:
    """Sampler + syndromes + observables for one code on one device."""

    def __init__(self, H_csr, priors, observables, device="cuda:0", seed: int = 0):
        self.device = torch.device(device)
        self.H = _DeviceCSR(sp.csr_matrix(H_csr), self.device)
        self.O = _DeviceCSR(sp.csr_matrix(observables), self.device)
        if self.H.N != self.O.N:
            raise ValueError("H and the observables matrix must have the same number of columns")
        self.V = self.H.N
        self.p = torch.from_numpy(np.asarray(priors, np.float32)).to(self.device)
        if self.p.numel() != self.V:
            raise ValueError("one prior per column")
        self.gen = torch.Generator(device=self.device)
        self.gen.manual_seed(int(seed))

    def sample(self, B: int):
        """(errors [B, V] uint8, syndromes [B, C] uint8) on the device."""
        e = (torch.rand(B, self.V, generator=self.gen, device=self.device) < self.p).to(torch.uint8)
        return e, self.H.apply(e)

    def failures(self, e: torch.Tensor, out: dict):
        """Device counts (failures, unconverged, logical flips) of one decoded batch."""
        flip = (self.O.apply(e) != self.O.apply(out["errors"].to(torch.uint8))).any(dim=1)
        unconv = out["found_count"] <= 0
        return torch.stack([(flip | unconv).sum(), unconv.sum(), (flip & ~unconv).sum(),
                            out["iterations"].to(torch.int64).sum()])

    def run(self, decode: Callable[[torch.Tensor], dict], shots: int, batch: int = 65536,
            warmup: bool = True) -> MCResult:
        """Decode `shots` fresh shots in batches with `decode`; counts stay on the device until the end.
        With ``warmup`` one extra batch of the same size is decoded first, untimed and uncounted
        (first-call costs: buffers, graph capture), from its own generator so the counted shots do
        not depend on it."""
        totals = torch.zeros(4, dtype=torch.int64, device=self.device)
        if warmup and shots > 0:
            g = torch.Generator(device=self.device)
            g.manual_seed(0x5EED)
            n = min(batch, shots)
            e = (torch.rand(n, self.V, generator=g, device=self.device) < self.p).to(torch.uint8)
            decode(self.H.apply(e))
        secs = 0.0
        done = 0
        while done < shots:
            n = min(batch, shots - done)
            e, s = self.sample(n)
            torch.cuda.synchronize(self.device)
            t0 = time.perf_counter()
            out = decode(s)
            torch.cuda.synchronize(self.device)
            secs += time.perf_counter() - t0
            totals += self.failures(e, out)
            done += n
        f, u, l, it = (int(x) for x in totals.cpu())
        return MCResult(shots=shots, failures=f, unconverged=u, logical_flips=l,
                        mean_iterations=it / shots if shots else 0.0, decode_seconds=secs)


def observables_for(workload) -> np.ndarray:
    """The workload's logical operators as a [k, V] matrix over all columns (data errors of every
    round accumulate)."""
    O = np.zeros((workload.logicals.shape[0], workload.H.shape[1]), np.uint8)
    for cols in workload.data_cols:
        O[:, cols] = workload.logicals
    return O


def main(argv=None):
    import argparse
    import json

    from . import codes
    from .decoder import RelayBPDecoder
    from .proposal import RELAY, LearnedRelayBPDecoder, ProposalNet, default_weights_path, load_params

    ap = argparse.ArgumentParser(prog="python -m pelagos_b200.montecarlo")
    ap.add_argument("--workload", default="bb144_phen")
    ap.add_argument("--p", type=float, default=0.003)
    ap.add_argument("--shots", type=int, default=1 << 20)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--decoder", choices=["plain", "learned"], default="plain")
    a = ap.parse_args(argv)
    w = codes.workload(a.workload, p=a.p)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    run = dec.decode
    if a.decoder == "learned":
        run = LearnedRelayBPDecoder(dec, ProposalNet(dec, load_params(default_weights_path(a.workload, a.p))[0]),
                                    gate=True).decode
    mc = MonteCarlo(w.H, w.priors, observables_for(w), seed=a.seed)
    res = mc.run(run, a.shots, a.batch)
    print(json.dumps({"workload": a.workload, "p": a.p, "decoder": a.decoder, **res.as_dict()}))


if __name__ == "__main__":
    main()
