"""Launch-shape autotuner for the decode kernel.

The kernel's shape is (group_threads, groups_per_block): how many threads share
one shot (and so how many variables and checks each thread owns), and how many
shots a thread block decodes at once.  ``tune`` times candidate shapes on a
sample batch with CUDA events and keeps the fastest.  The choice is cached in a
JSON file keyed by device name, graph sparsity hash, message type and the
decode parameters, in the way the reference keys its tuning cache
(src/pelagos/autotune.py:130-133, 222-541):

* cache file: ``$PELAGOS_B200_TUNE_CACHE`` or ``~/.cache/pelagos_b200_tune.json``;
* candidates: every warp multiple G from 32 to 1024 that gives at most 16
  variables and 32 checks per thread, each with the largest group count that
  fits (and, for one-warp groups, also half of it);
* a candidate the library rejects (shared memory, registers) is skipped.
"""

from __future__ import annotations

import json
import os
import threading
from pathlib import Path
from typing import Iterable, List, Optional, Tuple

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


def candidates(C: int, V: int) -> List[Tuple[int, int]]:
    out = []
    for G in range(32, 1025, 32):
        need = -(-V // G)
        if need > 16 or -(-C // G) > 32:
            continue
        out.append((G, 0))
        if G == 32:
            out.append((G, 8))
    return out


def lookup(dec, B: int) -> Optional[Tuple[int, int]]:
    v = _load().get(cache_key(dec, B))
    return tuple(v["shape"]) if v else None


def tune(dec, syndromes: torch.Tensor, shapes: Optional[Iterable[Tuple[int, int]]] = None, repeats: int = 2,
         use_cache: bool = True, verbose: bool = False) -> Tuple[int, int]:
    """Time the candidate shapes on `syndromes` (device tensor); configure and return the fastest."""
    B = int(syndromes.shape[0])
    key = cache_key(dec, B)
    if use_cache:
        hit = lookup(dec, B)
        if hit is not None:
            dec.configure_launch(*hit)
            return hit
    results = []
    shapes = list(shapes) if shapes is not None else candidates(dec.C, dec.V)
    for G, NG in shapes:
        try:
            dec.configure_launch(G, NG)
        except (NotImplementedError, ValueError):
            continue
        dec.decode(syndromes)  # warm-up
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dec.decode(syndromes)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        info = dec.launch_info()
        results.append((best, (info["group_threads"], info["groups_per_block"])))
        if verbose:
            print(f"  G={G:4d} groups={info['groups_per_block']:2d}: {best:8.3f} ms", flush=True)
    if not results:
        raise RuntimeError("no launch shape could be configured")
    ms, shape = min(results)
    dec.configure_launch(*shape)
    _store(key, {"shape": list(shape), "ms": ms, "sample_shots": B,
                 "tried": [[list(s), t] for t, s in sorted(results)]})
    return shape
