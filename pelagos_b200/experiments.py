"""Measurement runs beyond the single benchmark line.

``precision_sweep``: the same seeded shots and leg draws decoded with float16,
bfloat16, float32 and float64 messages (16-bit messages keep float32
posteriors, memory and sums; float64 computes everything in float64 and is
the high-precision run, checked bit for bit against the CPU oracle's float64
mode by the test suite).  Per precision and noise rate it reports the logical
error rate with its 95% Wilson interval, mean iterations, throughput, the
fraction of shots whose outputs equal the float64 run's, and the posterior
LLR error against float64 (max and RMS over the shots whose iteration count
matches the float64 run, so both posteriors come from the same iteration).

Usage: ``python -m pelagos_b200.experiments precision [--shots N] [--out FILE]``
"""

from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import codes
from .decoder import RelayBPDecoder

RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)


def wilson(k: int, n: int, z: float = 1.959964) -> tuple[float, float]:
    if n == 0:
        return (0.0, 1.0)
    p = k / n
    d = 1 + z * z / n
    c = (p + z * z / (2 * n)) / d
    h = z * math.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return (max(0.0, c - h), min(1.0, c + h))


def _decode(dec, syn_dev):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = dec.decode(syn_dev, return_last_posterior=True)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {k: v.cpu().numpy() for k, v in out.items() if isinstance(v, torch.Tensor)}, dt


def precision_sweep(shots: int = 131072, ps=(0.002, 0.003, 0.004), dtypes=("float64", "float32", "float16", "bfloat16"),
                    seed: int = 4242, device: int = 0) -> list[dict]:
    rows = []
    for p in ps:
        w = codes.workload("bb144_phen", p=p)
        err, syn = w.sample(shots, seed=seed)
        syn_dev = torch.from_numpy(syn).to(f"cuda:{device}")
        ref = None
        for dt in dtypes:
            dec = RelayBPDecoder(w.H, w.priors, data_type=dt, device=[device], **RELAY)
            _decode(dec, syn_dev[:1024])  # warm-up
            out, secs = _decode(dec, syn_dev)
            conv = out["found_count"] > 0
            fails = w.logical_failures(err, out["errors"], conv)
            lo, hi = wilson(int(fails.sum()), shots)
            row = {"p": p, "dtype": dt, "shots": shots, "ler": float(fails.mean()), "ler_ci95": [lo, hi],
                   "failures": int(fails.sum()), "unconverged": int((~conv).sum()),
                   "mean_iterations": float(out["iterations"].mean()), "shots_per_s": shots / secs}
            if dt == "float64":
                ref = out
            else:
                same_it = out["iterations"] == ref["iterations"]
                d = (out["last_posterior"].astype(np.float64) - ref["last_posterior"])[same_it]
                row.update({
                    "identical_errors_frac": float(np.mean(np.all(out["errors"] == ref["errors"], axis=1))),
                    "identical_iterations_frac": float(same_it.mean()),
                    "llr_err_max": float(np.abs(d).max()) if d.size else None,
                    "llr_err_rms": float(np.sqrt(np.mean(d * d))) if d.size else None,
                    "llr_ref_rms": float(np.sqrt(np.mean(ref["last_posterior"][same_it] ** 2))) if d.size else None,
                })
            rows.append(row)
            print(json.dumps(row), flush=True)
    return rows


def decode_case(shots: int, launch=(480, 1), learned: bool = False) -> None:
    """A small profiling case: two decodes of the same seeded [[144,12,12]] phenomenological batch
    (p = 0.003), with the plain decoder or the learned (gated) one run eagerly; either decode is
    two decode-kernel launches (pre-iterations, relay legs), the learned one with the network
    launch between them."""
    w = codes.workload("bb144_phen", p=0.003)
    syn = torch.from_numpy(w.sample(shots, seed=2026)[1]).cuda()
    dec = RelayBPDecoder(w.H, w.priors, launch=launch, **RELAY)
    run = dec.decode
    if learned:
        from .proposal import LearnedRelayBPDecoder, ProposalNet, default_weights_path, load_params

        run = LearnedRelayBPDecoder(dec, ProposalNet(dec, load_params(default_weights_path())[0]), gate=True,
                                    graph=False).decode
    for _ in range(2):
        out = run(syn)
    torch.cuda.synchronize()
    print(json.dumps({"shots": shots, "shot_iterations": int(out["iterations"].sum())}))


def markdown(rows: list[dict]) -> str:
    out = ["| p | messages | LER [95% CI] | unconverged | mean iters | shots/s | same errors as f64 | "
           "same iterations | LLR err max | LLR err RMS (ref RMS) |", "|---|---|---|---|---|---|---|---|---|---|"]
    for r in rows:
        ci = r["ler_ci95"]
        tail = ("— | — | — | —" if r["dtype"] == "float64" else
                f"{r['identical_errors_frac']:.5f} | {r['identical_iterations_frac']:.4f} | "
                f"{r['llr_err_max']:.3g} | {r['llr_err_rms']:.3g} ({r['llr_ref_rms']:.3g})")
        out.append(f"| {r['p']} | {r['dtype']} | {r['ler']:.2e} [{ci[0]:.1e}, {ci[1]:.1e}] | {r['unconverged']} | "
                   f"{r['mean_iterations']:.2f} | {r['shots_per_s']:.3g} | {tail} |")
    return "\n".join(out)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["precision", "decode-case"])
    ap.add_argument("--shots", type=int, default=131072)
    ap.add_argument("--launch", default="480,1",
                    help="decode-case: G,groups[,shots_per_group[,blocks_per_sm]] kernel shape")
    ap.add_argument("--learned", action="store_true", help="decode-case: the learned (gated, eager) decode")
    ap.add_argument("--out", default=None)
    ap.add_argument("--dtypes", default="float64,float32,float16,bfloat16",
                    help="comma-separated; float64 (the reference run) must come first")
    args = ap.parse_args(argv)
    if args.what == "decode-case":
        decode_case(args.shots, tuple(int(x) for x in args.launch.split(",")), learned=args.learned)
        return
    rows = precision_sweep(shots=args.shots, dtypes=tuple(args.dtypes.split(",")))
    md = markdown(rows)
    print(md)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
