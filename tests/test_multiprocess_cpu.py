"""The multi-GPU (replica) path's host logic on CPU: batch splitting and gathering across
replicas, the order of launches and host reads (every shard launches before any result is
read), a sharded decode over two gloo ranks gathered in order, and the benchmark's
max-over-ranks timing with two gloo ranks."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench
from pelagos_b200.decoder import RelayBPDecoder


@pytest.mark.parametrize("B,n", [(10, 3), (7, 7), (3, 5), (0, 2), (65536, 8)])
def test_split_batch_is_contiguous_and_balanced(B, n):
    parts = RelayBPDecoder._split_batch(B, n)
    assert len(parts) == n and parts[0][0] == 0 and parts[-1][1] == B
    assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
    sizes = [e - s for s, e in parts]
    assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def test_gather_offsets_unconverged_indices():
    dec = RelayBPDecoder.__new__(RelayBPDecoder)  # only the gather bookkeeping is exercised
    dec.device_ids = [0, 1]
    dec._device_strs = {0: "cpu", 1: "cpu"}
    splits = RelayBPDecoder._split_batch(5, 2)  # (0,3), (3,5)

    def part(n, unc):
        return {"errors": torch.zeros(n, 4, dtype=torch.uint8), "weights": torch.arange(n, dtype=torch.float32),
                "valid_mask": torch.ones(n, dtype=torch.bool), "iterations": torch.full((n,), 7, dtype=torch.int32),
                "found_count": torch.full((n,), 5, dtype=torch.int32),
                "unconverged_indices": torch.tensor(unc, dtype=torch.int32)}

    out = dec._gather([part(3, [1]), part(2, [0, 1])], splits)
    assert out["unconverged_indices"].tolist() == [1, 3, 4]
    assert out["weights"].tolist() == [0, 1, 2, 0, 1] and out["errors"].shape == (5, 4)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")  # the slowest replica: 15 ms
        dist.barrier()
        results[rank] = (ms, bench.whole_job_shots_per_s(world, 65536, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_replica():
    port = _free_port()
    with mp.Manager() as m:
        results = m.dict()
        mp.start_processes(_rank_main, args=(2, port, results), nprocs=2, join=True, start_method="spawn")
        got = dict(results)
    assert got[0] == got[1] == (15.0, 2 * 65536 / 0.015)


def test_without_a_process_group_the_value_is_local():
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def _fake_replica_decoder(monkeypatch, events):
    """A two-GPU RelayBPDecoder shell whose launch and finish steps only record their order."""
    dec = RelayBPDecoder.__new__(RelayBPDecoder)
    dec.__dict__.update(num_gpus=2, device_ids=[0, 1], _device_strs={0: "cpu", 1: "cpu"}, C=4, V=6,
                        perf="throughput", fast_max_unconverged_pct=None, hard_shots_first=True, num_sets=100,
                        pre_iter=80, _alpha_len=80, normalized_min_sum_alpha=None, stop_nconv=5)

    def launch(gpu_id, syn, *args, **kw):
        events.append(("launch", gpu_id, int(syn.shape[0])))
        return {"gpu_id": gpu_id, "n": int(syn.shape[0])}

    def finish(raw):
        events.append(("finish", raw["gpu_id"], raw["n"]))
        n = raw["n"]
        return {"errors": torch.zeros(n, 6, dtype=torch.uint8), "weights": torch.zeros(n),
                "valid_mask": torch.ones(n, dtype=torch.bool), "iterations": torch.ones(n, dtype=torch.int32),
                "found_count": torch.full((n,), 5, dtype=torch.int32),
                "unconverged_indices": torch.tensor([0], dtype=torch.int32)}

    monkeypatch.setattr(dec, "_launch_hard_first", launch)
    monkeypatch.setattr(dec, "_launch_on", launch)
    monkeypatch.setattr(dec, "_finish", finish)
    return dec


@pytest.mark.parametrize("B", [3000, 10])  # hard-shots-first shards, and plain single launches
def test_replica_shards_all_launch_before_any_host_read(monkeypatch, B):
    """Every device's kernels are enqueued before the first result is read back (a read
    synchronises the host), so the replicas decode concurrently."""
    events = []
    dec = _fake_replica_decoder(monkeypatch, events)
    out = dec.decode(torch.zeros(B, 4, dtype=torch.uint8))
    kinds = [e[0] for e in events]
    assert kinds == ["launch", "launch", "finish", "finish"]
    splits = RelayBPDecoder._split_batch(B, 2)
    assert [e[2] for e in events[:2]] == [e - s for s, e in splits]
    assert out["unconverged_indices"].tolist() == [0, splits[1][0]]  # offset by the shard start


def _shard_rank_main(rank: int, world: int, port: int, results):
    """One replica: decode its contiguous shard of a seeded batch with the CPU oracle standing in
    for its GPU, then gather every rank's results on every rank."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import oracle as O
        from pelagos_b200 import codes

        w = codes.workload("bb72_cc", p=0.08)
        err, syn = w.sample(96, seed=21)
        s0, s1 = RelayBPDecoder._split_batch(len(syn), world)[rank]
        legs = np.random.default_rng(3).uniform(-0.24, 0.66, (6, 72)).astype(np.float32)
        r = O.decode(O.reference_graph(w.H), syn[s0:s1], O.llr_from_priors(w.priors), pre_iter=10, num_sets=6,
                     set_max_iter=8, stop_nconv=3, gamma0=0.65, gamma_legs=legs, threads=1)
        part = {"errors": torch.from_numpy(r["errors"]), "weights": torch.from_numpy(r["weights"]),
                "valid_mask": torch.from_numpy(r["valid_mask"]), "iterations": torch.from_numpy(r["iterations"]),
                "found_count": torch.from_numpy(r["found_count"]),
                "unconverged_indices": torch.from_numpy(np.nonzero(r["found_count"] < 3)[0].astype(np.int32))}
        parts = [None] * world
        dist.all_gather_object(parts, part)
        dec = RelayBPDecoder.__new__(RelayBPDecoder)
        dec.device_ids = list(range(world))
        dec._device_strs = {i: "cpu" for i in range(world)}
        out = dec._gather(parts, RelayBPDecoder._split_batch(len(syn), world))
        results[rank] = {k: v.numpy() for k, v in out.items()}
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_sharded_decodes():
    """A sharded decode over two ranks (contiguous shards, gathered in order, unconverged indices
    offset by each shard's start) equals the single-process decode of the whole batch."""
    from oracle import oracle as O
    from pelagos_b200 import codes

    port = _free_port()
    with mp.Manager() as m:
        results = m.dict()
        mp.start_processes(_shard_rank_main, args=(2, port, results), nprocs=2, join=True, start_method="spawn")
        got = dict(results)
    w = codes.workload("bb72_cc", p=0.08)
    err, syn = w.sample(96, seed=21)
    legs = np.random.default_rng(3).uniform(-0.24, 0.66, (6, 72)).astype(np.float32)
    r = O.decode(O.reference_graph(w.H), syn, O.llr_from_priors(w.priors), pre_iter=10, num_sets=6,
                 set_max_iter=8, stop_nconv=3, gamma0=0.65, gamma_legs=legs, threads=1)
    for rank in (0, 1):
        np.testing.assert_array_equal(got[rank]["errors"], r["errors"])
        np.testing.assert_array_equal(got[rank]["iterations"], r["iterations"])
        np.testing.assert_array_equal(got[rank]["unconverged_indices"], np.nonzero(r["found_count"] < 3)[0])
