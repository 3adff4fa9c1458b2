"""Launch-shape autotuner for the decode kernel.

The kernel's shape is (group_threads, groups_per_block, shots_per_group[,
blocks_per_sm]): how many threads share one shot (and so how many variables
and checks each thread owns), how many groups a thread block holds, how many
shots a group decodes at once (1: relaybp_decode_kernel; 2: relaybp_slots_kernel,
one group per block), and for one-shot block-per-group launches how many
blocks the kernel is compiled to keep resident per SM (2: half the register
file each, two shots side by side with their own barriers).  The launches
that run only the pre-iterations may have their own shape (``kind="pre"``).  ``tune`` times candidate shapes on a sample batch with CUDA events
(the median of ``repeats`` timed runs after a warm-up, by default of
``decoder.decode`` and optionally of any decode call, e.g. a learned decode)
and keeps the fastest.  The choice is cached in a JSON file keyed by device
name, graph sparsity hash, message type and the decode parameters, in the way
the reference keys its tuning cache (src/pelagos/autotune.py:130-133, 222-541):

* cache file: ``$PELAGOS_B200_TUNE_CACHE`` or ``~/.cache/pelagos_b200_tune.json``;
* candidates: every warp multiple G from 32 to 1024 that gives at most 16
  variables and 32 checks per thread, with the multi-group kernel (the largest
  group count that fits and, for one-warp groups, also 8) and with the
  block-per-group kernel (one and two shots per group, and one shot per group
  at two resident blocks per SM);
* a candidate the library rejects (shared memory, registers) is skipped.

``default_shape`` returns the shape measured best for a workload and
committed with the package (``data/launch_shapes.json``, keyed by graph
sparsity hash and message type; ``default_pre_shape`` the pre-iteration
launches' shape where the entry gives one, and ``apply_default_shapes``
configures both), so a fresh machine starts from a measured shape instead of
re-tuning on a noisy sample.
"""

from __future__ import annotations

import json
import os
import threading
from pathlib import Path
from typing import Callable, Iterable, List, Optional, Tuple

import numpy as np
import torch

_LOCK = threading.Lock()
VPT_CHOICES = (1, 2, 3, 4, 6, 8, 12, 16)


def cache_path() -> Path:
    return Path(os.environ.get("PELAGOS_B200_TUNE_CACHE", Path.home() / ".cache" / "pelagos_b200_tune.json"))


def cache_key(dec, B: int) -> str:
    dev = torch.cuda.get_device_name(dec.device_ids[0])
    bucket = 1 << max(0, int(B - 1).bit_length())
    return "|".join(str(x) for x in (
        dev, dec.graph.sparsity_hash, dec.dtype_str, dec.pre_iter, dec.num_sets, dec.set_max_iter,
        dec.stop_nconv, dec.algo, f"B<={bucket}"))


def _load() -> dict:
    try:
        return json.loads(cache_path().read_text())
    except (OSError, ValueError):
        return {}


def _store(key: str, value) -> None:
    with _LOCK:
        data = _load()
        data[key] = value
        p = cache_path()
        try:
            p.parent.mkdir(parents=True, exist_ok=True)
            tmp = p.with_suffix(".tmp")
            tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
            tmp.replace(p)
        except OSError:
            pass  # a read-only home only loses the cache


def candidates(C: int, V: int) -> List[Tuple[int, int, int]]:
    out = []
    for ns in (1, 2):
        for G in range(32, 1025, 32):
            need = -(-V // G)
            if need > 16 or -(-C // G) > 32:
                continue
            if ns == 1:
                out.append((G, 0, 1))   # several one-shot groups per block, as many as fit
                if G == 32:
                    out.append((G, 8, 1))
            out.append((G, 1, ns))      # the block-per-group kernel
            if ns == 1 and G <= 512:
                out.append((G, 1, 1, 2))  # the same, compiled for two resident blocks per SM
    return out


def lookup(dec, B: int) -> Optional[Tuple[int, ...]]:
    v = _load().get(cache_key(dec, B))
    return tuple(v["shape"]) if v else None


SHAPES_FILE = Path(__file__).resolve().parent / "data" / "launch_shapes.json"


def _committed(dec) -> Optional[dict]:
    try:
        table = json.loads(SHAPES_FILE.read_text())
    except (OSError, ValueError):
        return None
    return table.get(f"{dec.graph.sparsity_hash}|{dec.dtype_str}")


def default_shape(dec) -> Optional[Tuple[int, ...]]:
    """The committed shape for this graph and message type, or None."""
    v = _committed(dec)
    return tuple(v["shape"]) if v else None


def default_pre_shape(dec) -> Optional[Tuple[int, ...]]:
    """The committed shape of the pre-iteration launches, or None (they use ``default_shape``)."""
    v = _committed(dec)
    return tuple(v["pre_shape"]) if v and "pre_shape" in v else None


def apply_default_shapes(dec) -> bool:
    """Configure the committed shapes of this workload; False when none is committed."""
    shape = default_shape(dec)
    if shape is None:
        return False
    dec.configure_launch(*shape)
    pre = default_pre_shape(dec)
    if pre is not None:
        dec.configure_launch(*pre, kind="pre")
    return True


def _time(fn: Callable[[], object], repeats: int) -> float:
    """Median of `repeats` event-timed calls after one warm-up call."""
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def tune(dec, syndromes: torch.Tensor, shapes: Optional[Iterable[Tuple[int, ...]]] = None, repeats: int = 5,
         use_cache: bool = True, verbose: bool = False,
         decode_fn: Optional[Callable[[torch.Tensor], object]] = None, kind: str = "all") -> Tuple[int, ...]:
    """Time the candidate shapes on `syndromes` (device tensor) with ``decode_fn`` (default
    ``dec.decode``); configure and return the fastest (median of ``repeats`` runs).  ``kind``
    "pre" or "legs" tunes only that launch kind's shape, the other kind keeping its own."""
    B = int(syndromes.shape[0])
    key = cache_key(dec, B) + ("" if decode_fn is None else "|custom") + ("" if kind == "all" else f"|{kind}")
    if use_cache and decode_fn is None and kind == "all":
        hit = lookup(dec, B)
        if hit is not None:
            dec.configure_launch(*hit)
            return hit
    fn = decode_fn or dec.decode
    results = []
    shapes = list(shapes) if shapes is not None else candidates(dec.C, dec.V)
    for shape in shapes:
        try:
            dec.configure_launch(*shape, kind=kind)
        except (NotImplementedError, ValueError):
            continue
        ms = _time(lambda: fn(syndromes), repeats)
        info = dec.launch_info()
        if kind == "pre":
            info = info["pre"]
        got = (info["group_threads"], info["groups_per_block"], info["shots_per_group"], info["blocks_per_sm"])
        results.append((ms, got))
        if verbose:
            print(f"  G={got[0]:4d} groups={got[1]:2d} shots/group={got[2]} blocks/SM={got[3]}: {ms:8.3f} ms",
                  flush=True)
    if not results:
        raise RuntimeError("no launch shape could be configured")
    ms, shape = min(results)
    dec.configure_launch(*shape, kind=kind)
    _store(key, {"shape": list(shape), "ms": ms, "sample_shots": B,
                 "tried": [[list(s), t] for t, s in sorted(results)]})
    return shape


def tune_mixed(mix, syndromes, repeats: int = 3, rounds: int = 2, verbose: bool = False) -> List[int]:
    """Per-code group sizes of a mixed launch (``MixedDecoder``): coordinate descent, one code
    at a time over the group sizes the launch's block size allows (multiples of 32 dividing it;
    the library rejects sizes whose threads would own too many variables or checks), each
    candidate timed as the median of ``repeats`` decodes of ``syndromes`` (one batch per code).
    Configures and returns the fastest sizes."""
    T = mix.launch_info()[0]["block_threads"]
    shapes = [x["group_threads"] for x in mix.launch_info()]
    best = _time(lambda: mix.decode(syndromes), repeats)
    if verbose:
        print(f"  start {shapes}: {best:8.3f} ms", flush=True)
    for _ in range(rounds):
        improved = False
        for i in range(len(shapes)):
            for G in range(32, T + 1, 32):
                if T % G or G == shapes[i]:
                    continue
                trial = list(shapes)
                trial[i] = G
                try:
                    mix.configure(trial)
                except (NotImplementedError, ValueError):
                    continue
                ms = _time(lambda: mix.decode(syndromes), repeats)
                if verbose:
                    print(f"  {trial}: {ms:8.3f} ms", flush=True)
                if ms < best:
                    best, shapes, improved = ms, trial, True
            mix.configure(shapes)
        if not improved:
            break
    mix.configure(shapes)
    return shapes
