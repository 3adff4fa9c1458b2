"""On-GPU Monte-Carlo loop: device sampling, syndromes and observables against the host
computation of the same shots."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from pelagos_b200 import RelayBPDecoder, codes
from pelagos_b200.montecarlo import MonteCarlo, observables_for

pytestmark = pytest.mark.gpu

RELAY = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=5, algo="relay", seed=1234)


@pytest.mark.parametrize("name,p", [("bb144_phen", 0.005), ("bb72_cc", 0.07)])
def test_counts_match_the_host(name, p):
    w = codes.workload(name, p=p)
    mc = MonteCarlo(w.H, w.priors, observables_for(w), seed=5)
    e, s = mc.sample(4096)
    e_h, s_h = e.cpu().numpy(), s.cpu().numpy()
    np.testing.assert_array_equal(s_h, (w.H @ e_h.T.astype(np.int64) % 2).T)
    assert abs(e_h.mean() - p) < 0.1 * p
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    out = dec.decode(s)
    got = mc.failures(e, out).cpu().numpy()
    o = {k: v.cpu().numpy() for k, v in out.items() if isinstance(v, torch.Tensor)}
    conv = o["found_count"] > 0
    fails = w.logical_failures(e_h, o["errors"], conv)
    assert got[0] == fails.sum() and got[1] == (~conv).sum()
    assert got[2] == (fails & conv).sum() and got[3] == o["iterations"].astype(np.int64).sum()
    if name == "bb72_cc":  # failures are a few percent there; the phenomenological code may have none
        assert got[0] > 0


def test_runs_are_seeded():
    w = codes.workload("bb72_cc", p=0.07)
    dec = RelayBPDecoder(w.H, w.priors, **RELAY)
    a = MonteCarlo(w.H, w.priors, observables_for(w), seed=9).run(dec.decode, 3000, batch=1024)
    b = MonteCarlo(w.H, w.priors, observables_for(w), seed=9).run(dec.decode, 3000, batch=1024)
    assert (a.failures, a.unconverged, a.mean_iterations) == (b.failures, b.unconverged, b.mean_iterations)
    assert a.shots == 3000 and 0 < a.ler < 1 and a.ler_ci95[0] <= a.ler <= a.ler_ci95[1]
