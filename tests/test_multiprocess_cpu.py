"""The multi-GPU (replica) path's host logic on CPU: batch splitting and gathering across
replicas, and the benchmark's max-over-ranks timing with two gloo ranks."""

from __future__ import annotations

import os
import socket

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
