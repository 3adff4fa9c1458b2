"""Generate golden input/output vectors by running the reference decoder itself.

The reference (quantum-supercomputing/pelagos) is Python + Triton.  Its decoder
insists on a CUDA device, so this script runs it on the CPU instead:

* ``TRITON_INTERPRET=1`` makes every ``@triton.jit`` kernel of
  ``src/pelagos/kernels.py`` execute through Triton's numpy interpreter, so the
  arithmetic is the kernels' own, evaluated in IEEE float32 with one rounding
  per operation;
* a ``TorchFunctionMode`` maps every ``cuda`` device argument to ``cpu`` and
  ``torch.cuda.device`` becomes a no-op context;
* the autotuner is replaced, exactly as the reference's own test fixture
  ``fixed_launch_configs`` does (tests/test_decoder_fixes.py:145-156), by the
  first candidate configuration of each kernel;
* the seeded leg draws of ``sample_gamma_uniform`` / ``sample_gamma_per_variable``
  (src/pelagos/utils.py:128-225) run on a CPU ``torch.Generator``.  Their values
  therefore differ from a CUDA draw, so every draw is recorded in the fixture
  and replayed as an explicit table by the code under test.

Each case is written to ``tests/golden/<case>.npz`` with the check matrix, the
priors, the syndromes, every constructor / decode argument, the gamma rows the
legs used, the reference's variable-edge order (``var_edges``, built with a
non-stable ``np.argsort`` in src/pelagos/graph.py:145) and the decode outputs.

This script imports the reference from the directory named by the environment
variable ``PELAGOS_REF_SRC`` (the ``src`` directory of a pelagos checkout) and so
only runs where such a tree exists; the fixtures it writes are what the tests
consume.

Usage: ``PELAGOS_REF_SRC=<pelagos>/src python tests/golden/make_golden.py [case ...]``
(default: all cases).
"""

from __future__ import annotations

import json
import os
import sys
import time
from pathlib import Path

os.environ["TRITON_INTERPRET"] = "1"
REF_SRC = os.environ.get("PELAGOS_REF_SRC")
if not REF_SRC or not Path(REF_SRC, "pelagos", "decoder.py").exists():
    raise SystemExit("set PELAGOS_REF_SRC to the src directory of a pelagos checkout")
sys.path.insert(0, REF_SRC)

import numpy as np  # noqa: E402
import torch  # noqa: E402
from scipy.sparse import csr_matrix  # noqa: E402
from torch.overrides import TorchFunctionMode  # noqa: E402

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
from pelagos_b200 import codes  # noqa: E402


def _cpu(d):
    if isinstance(d, str) and d.startswith("cuda"):
        return "cpu"
    if isinstance(d, torch.device) and d.type == "cuda":
        return torch.device("cpu")
    return d


class _CpuMode(TorchFunctionMode):
    def __torch_function__(self, func, types, args=(), kwargs=None):
        kwargs = dict(kwargs or {})
        if "device" in kwargs:
            kwargs["device"] = _cpu(kwargs["device"])
        args = tuple(_cpu(a) for a in args)
        return func(*args, **kwargs)


class _NoDevice:
    def __init__(self, *a, **k):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def _patch_reference():
    torch.cuda.is_available = lambda: True
    torch.cuda.device_count = lambda: 1
    torch.cuda.device = _NoDevice
    import pelagos.decoder as dmod

    draws: list[np.ndarray] = []
    orig_u = dmod.sample_gamma_uniform
    orig_pv = dmod.sample_gamma_per_variable

    def sgu(rows, V, lo, hi, device, seed=None):
        g = orig_u(rows, V, lo, hi, "cpu", seed)
        draws.append(g.float().numpy().copy())
        return g

    def spv(rows, V, intervals, device, seed=None):
        g = orig_pv(rows, V, intervals, "cpu", seed)
        draws.append(g.float().numpy().copy())
        return g

    dmod.sample_gamma_uniform = sgu
    dmod.sample_gamma_per_variable = spv
    chosen: dict = {}

    def fixed(self, *, kernel_name, build_cfgs_fn, **kwargs):
        if kernel_name not in chosen:
            c = build_cfgs_fn()[0]
            chosen[kernel_name] = dict(c.kwargs, num_warps=c.num_warps, num_stages=c.num_stages)
        return dict(chosen[kernel_name])

    dmod.RelayBPDecoder._get_tuned_meta = fixed
    return dmod, draws


# ----------------------------------------------------------------------------- cases

DET = dict(pre_iter=200, num_sets=1, set_max_iter=0, gamma0=0.0,
           gamma_dist_interval=(0.0, 1e-12), stop_nconv=1, normalized_min_sum_alpha=1.0,
           data_type="float32", algo="plain", seed=1234)


def _small_random(n, c, seed):
    """tests/test_triton_against_rust.py:440-452 construction."""
    rng = np.random.default_rng(seed)
    Hd = np.zeros((c, n), dtype=np.uint8)
    for i in range(c):
        deg = int(rng.integers(2, min(4, n) + 1))
        cols = rng.choice(n, size=deg, replace=False)
        Hd[i, cols] = 1
    H = csr_matrix(Hd)
    H.sort_indices()
    p = np.clip(rng.uniform(0.005, 0.02, size=n).astype(np.float64), 1e-6, 1 - 1e-6)
    S = np.stack([rng.integers(0, 2, size=c, dtype=np.uint8) for _ in range(8)])
    return H, p, S


def _problem24x40(B=24):
    """tests/test_unconverged_correction.py:41-53 construction."""
    rng = np.random.default_rng(7)
    Hd = np.zeros((24, 40), dtype=np.uint8)
    for c in range(24):
        for v in rng.choice(40, 4, replace=False):
            Hd[c, v] = 1
    syn = np.random.default_rng(3).integers(0, 2, size=(B, 24)).astype(np.uint8)
    return csr_matrix(Hd), np.full(40, 0.06), syn


def _bb72_case(B, p=0.05, seed=11):
    H = codes.bb_code_capacity_72()
    rng = np.random.default_rng(seed)
    e = (rng.random((B, H.shape[1])) < p).astype(np.uint8)
    s = ((H @ e.T) % 2).T.astype(np.uint8)
    return H, np.full(H.shape[1], p), s


def _cases():
    cases = {}
    tri3 = csr_matrix(np.array([[1, 1, 0], [0, 1, 1], [1, 0, 1]], dtype=np.uint8))
    syn8 = np.array([[(x >> i) & 1 for i in range(3)] for x in range(8)], dtype=np.uint8)
    cases["triangle_relay"] = lambda: (
        tri3, np.full(3, 0.05), syn8,
        dict(pre_iter=10, num_sets=2, set_max_iter=10, stop_nconv=1, data_type="float32",
             algo="relay"), {})
    tri2 = csr_matrix(np.array([[1, 1, 0], [0, 1, 1]], dtype=np.uint8))
    cases["triangle_det"] = lambda: (
        tri2, np.array([0.01, 0.01, 0.01]),
        np.array([[0, 0], [1, 0], [0, 1], [1, 1]], np.uint8), dict(DET), {})
    for (n, c, sd) in [(8, 4, 0), (10, 5, 1)]:
        def mk(n=n, c=c, sd=sd):
            H, p, S = _small_random(n, c, sd)
            return H, p, S, dict(DET), {}
        cases[f"random_{n}x{c}_det"] = mk

    def high_degree():
        Hd = np.zeros((3, 25), dtype=np.uint8)
        Hd[0, :20] = 1
        Hd[1, 5:15] = 1
        Hd[2, [0, 10, 20]] = 1
        S = np.array([[1, 0, 1], [1, 1, 0], [0, 1, 1], [1, 1, 1]], np.uint8)
        return csr_matrix(Hd), np.full(25, 0.01), S, dict(DET), {}
    cases["high_degree_det"] = high_degree

    def chain5():
        Hd = np.array([[1, 1, 0, 0, 0], [0, 1, 1, 0, 0], [0, 0, 1, 1, 0], [0, 0, 0, 1, 1]], np.uint8)
        S = np.array([[1, 0, 1, 0], [1, 1, 1, 1], [0, 1, 0, 1], [1, 0, 0, 1]], np.uint8)
        kw = dict(DET, gamma0=0.1, pre_iter=10, num_sets=2, set_max_iter=5,
                  gamma_dist_interval=(0.0, 0.2), stop_nconv=2, seed=42)
        return csr_matrix(Hd), np.full(5, 0.01), S, kw, {}
    cases["chain5_ensemble"] = chain5

    def nonconv():
        Hd = np.array([[1, 1, 1, 1, 0, 0], [0, 1, 1, 0, 1, 1], [1, 0, 1, 0, 1, 1]], np.uint8)
        kw = dict(DET, set_max_iter=0, num_sets=1, stop_nconv=1)
        return csr_matrix(Hd), np.full(6, 0.5), np.array([[1, 1, 1]], np.uint8), kw, {}
    cases["uninformative_det"] = nonconv

    def unsorted():
        H = csr_matrix(np.array([[1, 0, 1, 0], [0, 1, 1, 1]], np.uint8))
        Hu = csr_matrix((H.data, H.indices[::-1], H.indptr), shape=H.shape)
        S = np.array([[1, 0], [0, 1], [1, 1]], np.uint8)
        return Hu, np.array([0.02, 0.01, 0.03, 0.02]), S, dict(DET), {}
    cases["unsorted_csr_det"] = unsorted

    base24 = dict(pre_iter=4, num_sets=3, set_max_iter=4, gamma0=0.1, stop_nconv=1,
                  seed=42, algo="relay", data_type="float32")
    cases["rand24x40_first_leg"] = lambda: (*_problem24x40(), dict(base24), {})
    cases["rand24x40_last_leg"] = lambda: (
        *_problem24x40(), dict(base24, unconverged_correction="last_leg"), {})
    cases["rand24x40_pre0"] = lambda: (*_problem24x40(), dict(base24, pre_iter=0), {})
    cases["rand24x40_S2"] = lambda: (*_problem24x40(), dict(base24, stop_nconv=2), {})
    cases["rand24x40_plain"] = lambda: (*_problem24x40(), dict(base24, algo="plain"), {})
    cases["rand24x40_numsets0"] = lambda: (*_problem24x40(), dict(base24, num_sets=0), {})

    bbkw = dict(pre_iter=20, num_sets=4, set_max_iter=10, stop_nconv=2, algo="relay",
                data_type="float32", seed=1234)
    cases["bb72_relay_S2"] = lambda: (*_bb72_case(8), dict(bbkw), {})
    cases["bb72_alpha_ramp"] = lambda: (
        *_bb72_case(8, seed=12), dict(bbkw, normalized_min_sum_alpha=0.0, stop_nconv=3), {})
    cases["bb72_alpha08"] = lambda: (
        *_bb72_case(8, seed=13), dict(bbkw, normalized_min_sum_alpha=0.8), {})
    cases["bb72_beta"] = lambda: (
        *_bb72_case(8, seed=14), dict(bbkw, offset_min_sum_beta=0.25), {})

    def bb72_explicit():
        H, p, s = _bb72_case(8, seed=15)
        g = np.random.default_rng(6).uniform(-0.24, 0.66, (3, H.shape[1])).astype(np.float32)
        return H, p, s, dict(bbkw, explicit_gammas=g, num_sets=5), {}
    cases["bb72_explicit"] = bb72_explicit

    def bb72_by_error():
        H, p, s = _bb72_case(8, seed=16)
        V = H.shape[1]
        iv = np.stack([np.full(V, -0.3), np.linspace(0.3, 0.8, V)], axis=1).astype(np.float32)
        return H, p, s, dict(bbkw, gamma_dist_interval_by_error=iv), {}
    cases["bb72_by_error"] = bb72_by_error

    def bb72_resume():
        H, p, s = _bb72_case(8, seed=17)
        V = H.shape[1]
        rng = np.random.default_rng(18)
        init_post = (2.944439 + rng.normal(0, 1.0, (8, V))).astype(np.float32)
        init_gamma = rng.uniform(0.0, 0.9, (8, V)).astype(np.float32)
        prior = (rng.uniform(2.0, 4.0, (8, V))).astype(np.float32)
        dkw = dict(init_posterior=init_post, init_gamma=init_gamma, prior_llr=prior,
                   pre_iter_override=12, return_last_posterior=True)
        return H, p, s, dict(bbkw), dkw
    cases["bb72_resume"] = bb72_resume

    def bb72_skip_legs():
        H, p, s = _bb72_case(8, seed=19)
        return H, p, s, dict(bbkw, pre_iter=6), dict(skip_relay_legs=True,
                                                    return_last_posterior=True)
    cases["bb72_skip_legs"] = bb72_skip_legs
    cases["bb72_fp64"] = lambda: (*_bb72_case(8, seed=20), dict(bbkw, data_type="float64"), {})

    def regular_pre3():
        H = codes.regular_ldpc(C=300, V=600, seed=3)
        V = H.shape[1]
        pr = np.random.default_rng(4).uniform(0.01, 0.03, V)
        E = (np.random.default_rng(5).random((16, V)) < pr * 3.0).astype(np.uint8)
        S = ((H @ E.T) % 2).T.astype(np.uint8)
        kw = dict(pre_iter=3, num_sets=0, set_max_iter=20, stop_nconv=1, gamma0=0.65,
                  algo="relay", data_type="float32", seed=7)
        return H, pr, S, kw, dict(skip_relay_legs=True, return_last_posterior=True)
    cases["regular300x600_pre3"] = regular_pre3

    # The full Relay-BP-S schedule of every benchmark configuration (pre 80, 100 legs of at most
    # 60 iterations, gamma0 0.65, U(-0.24, 0.66) legs, stop_nconv 5: decoder.py:271-307 defaults).
    full = dict(pre_iter=80, num_sets=100, set_max_iter=60, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
                stop_nconv=5, algo="relay", data_type="float32", seed=1234)
    cases["bb72_full_schedule"] = lambda: (*_bb72_case(6, seed=31), dict(full), {})
    cases["bb72_full_schedule_plain"] = lambda: (*_bb72_case(4, seed=32), dict(full, algo="plain"), {})

    def bb144_phen(B, p, seed):
        w = codes.workload("bb144_phen", p=p)
        err, syn = w.sample(B, seed=seed)
        return w.H, w.priors, syn

    # the benchmark's [[144,12,12]] phenomenological matrix (936 x 2592) with a short schedule
    cases["bb144_phen_short"] = lambda: (
        *bb144_phen(2, 0.004, 41),
        dict(pre_iter=6, num_sets=2, set_max_iter=4, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=2, algo="relay", data_type="float32", seed=1234), {})
    cases["bb144_phen_dense"] = lambda: (
        *bb144_phen(2, 0.012, 43),
        dict(pre_iter=12, num_sets=3, set_max_iter=6, gamma0=0.65, gamma_dist_interval=(-0.24, 0.66),
             stop_nconv=3, algo="relay", data_type="float32", seed=1234), {})
    return cases


def run_case(name: str, build) -> Path:
    dmod, draws = _patch_reference()
    from pelagos import RelayBPDecoder

    H, priors, S, kw, dkw = build()
    H = csr_matrix(H)
    t0 = time.time()
    with _CpuMode():
        dec = RelayBPDecoder(H_csr=H, error_priors=np.asarray(priors, np.float64), **kw)
        dargs = {}
        for k, v in dkw.items():
            dargs[k] = torch.from_numpy(np.asarray(v)) if isinstance(v, np.ndarray) else v
        out = dec.decode(torch.from_numpy(np.asarray(S, np.uint8)), **dargs)
    g = dec.graphs[0]
    arrays = dict(
        indptr=H.indptr.astype(np.int32), indices=H.indices.astype(np.int32),
        shape=np.array(H.shape, np.int64), priors=np.asarray(priors, np.float64),
        syndromes=np.asarray(S, np.uint8),
        ref_var_ptr=g.var_ptr.numpy().astype(np.int32),
        ref_var_edges=g.var_edges.numpy().astype(np.int32),
        ref_edge_var=g.edge_var.numpy().astype(np.int32),
        leg_draws=(np.concatenate(draws, axis=0) if draws else np.zeros((0, H.shape[1]), np.float32)),
        out_errors=out["errors"].numpy().astype(np.uint8),
        out_weights=out["weights"].float().numpy(),
        out_valid_mask=out["valid_mask"].numpy(),
        out_iterations=out["iterations"].numpy().astype(np.int32),
        out_found_count=out["found_count"].numpy().astype(np.int32),
        out_unconverged_indices=out["unconverged_indices"].numpy().astype(np.int32),
    )
    if "last_posterior" in out:
        arrays["out_last_posterior"] = out["last_posterior"].double().numpy()
    meta_kw = {}
    for k, v in kw.items():
        if isinstance(v, np.ndarray):
            arrays["kw_" + k] = v
        else:
            meta_kw[k] = list(v) if isinstance(v, tuple) else v
    meta_dkw = {}
    for k, v in dkw.items():
        if isinstance(v, np.ndarray):
            arrays["dkw_" + k] = v
        else:
            meta_dkw[k] = v
    arrays["meta"] = np.array(json.dumps({"kwargs": meta_kw, "decode_kwargs": meta_dkw,
                                           "generator": "pelagos under TRITON_INTERPRET=1",
                                           "seconds": round(time.time() - t0, 1)}))
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    return path


def main(argv):
    cases = _cases()
    names = argv or list(cases)
    for n in names:
        t = time.time()
        p = run_case(n, cases[n])
        print(f"{n}: {time.time() - t:.1f}s -> {p.name}", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
