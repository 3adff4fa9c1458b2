"""ctypes front end of the CPU oracle (oracle/relaybp_oracle.cpp).  TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, as the checker.  The decoder package never
imports it.

``decode`` takes the reference's graph arrays and the same per-call options as
``RelayBPDecoder.decode`` and returns numpy arrays.  The leg gamma table must be
supplied explicitly (see ``leg_table``) because the reference draws it on the
device with torch's generator.
"""

from __future__ import annotations

import ctypes as ct
import os
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

MSG_TYPES = {"float32": 0, "float16": 1, "bfloat16": 2, "float64": 3}
MIX_MODES = {"separate": 0, "fma_gp": 1, "fma_lp": 2}


class _Params(ct.Structure):
    _fields_ = [("pre_iter", ct.c_int32), ("num_sets", ct.c_int32), ("set_max_iter", ct.c_int32),
                ("stop_nconv", ct.c_int32), ("last_leg", ct.c_int32), ("use_alpha", ct.c_int32),
                ("use_beta", ct.c_int32), ("beta", ct.c_float), ("mix_mode", ct.c_int32),
                ("msg_type", ct.c_int32), ("skip_relay_legs", ct.c_int32), ("num_threads", ct.c_int32)]


class _Graph(ct.Structure):
    _fields_ = [("C", ct.c_int32), ("V", ct.c_int32), ("E", ct.c_int32), ("chk_ptr", ct.c_void_p),
                ("edge_var", ct.c_void_p), ("var_ptr", ct.c_void_p), ("var_edges", ct.c_void_p)]


class _Inputs(ct.Structure):
    _fields_ = [("B", ct.c_int64), ("syndromes", ct.c_void_p), ("llr", ct.c_void_p),
                ("llr_per_shot", ct.c_void_p), ("gamma0", ct.c_float), ("gamma_pre", ct.c_void_p),
                ("gamma_legs", ct.c_void_p), ("gamma_legs_shot", ct.c_void_p),
                ("n_shot_legs", ct.c_int32), ("init_posterior", ct.c_void_p),
                ("alpha_table", ct.c_void_p)]


class _Outputs(ct.Structure):
    _fields_ = [("errors", ct.c_void_p), ("weights", ct.c_void_p), ("weight_fixed", ct.c_void_p),
                ("found_count", ct.c_void_p), ("iterations", ct.c_void_p),
                ("last_posterior", ct.c_void_p)]


_lib = None


def build() -> Path:
    """Compile the oracle with oracle/Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < (HERE / "relaybp_oracle.cpp").stat().st_mtime:
            build()
        _lib = ct.CDLL(str(LIB))
        _lib.rbo_decode.restype = ct.c_int
        _lib.rbo_decode.argtypes = [ct.POINTER(_Graph), ct.POINTER(_Params), ct.POINTER(_Inputs),
                                    ct.POINTER(_Outputs)]
        for f in (_lib.rbo_round_f16, _lib.rbo_round_bf16):
            f.restype = None
            f.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int64]
    return _lib


def _p(a):
    return ct.c_void_p(a.ctypes.data) if a is not None else ct.c_void_p(0)


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(np.asarray(a), dtype=dt)


def round_f16(x: np.ndarray) -> np.ndarray:
    x = _c(x, np.float32)
    y = np.empty_like(x)
    lib().rbo_round_f16(_p(x), _p(y), x.size)
    return y


def round_bf16(x: np.ndarray) -> np.ndarray:
    x = _c(x, np.float32)
    y = np.empty_like(x)
    lib().rbo_round_bf16(_p(x), _p(y), x.size)
    return y


def reference_graph(H) -> dict:
    """Edge-centric arrays exactly as src/pelagos/graph.py:101-211 builds them."""
    from scipy.sparse import csr_matrix, issparse

    if not issparse(H):
        H = csr_matrix(np.asarray(H))
    H = H.tocsr()
    if H.dtype != np.uint8 and H.dtype != bool:
        H = (H != 0).astype(np.uint8)
    C, V = H.shape
    chk_ptr = H.indptr.astype(np.int32)
    edge_var = H.indices.astype(np.int32)
    var_edges = np.argsort(edge_var).astype(np.int32)
    var_ptr = np.zeros(V + 1, np.int32)
    np.cumsum(np.bincount(edge_var, minlength=V), out=var_ptr[1:])
    return {"C": C, "V": V, "E": int(H.nnz), "chk_ptr": chk_ptr, "edge_var": edge_var,
            "var_ptr": var_ptr, "var_edges": var_edges}


def alpha_table(alpha: Optional[float], scaling: float, n: int) -> tuple[bool, np.ndarray]:
    """Per-iteration alpha as decoder.py:2648-2660 computes it (float64, then float32)."""
    n = max(int(n), 1)
    if alpha is None:
        return False, np.ones(n, np.float32)
    a = float(alpha)
    if a == 0.0:
        s = float(scaling or 1.0)
        return True, np.array([1.0 - 2.0 ** (-((t + 1) / s)) for t in range(n)], np.float32)
    return True, np.full(n, 1.0 if a < 0 else a, np.float32)


def llr_from_priors(priors) -> np.ndarray:
    """utils.py:88-107: clip to [1e-10, 0.5-1e-10], log((1-p)/p) in float64, then float32."""
    p = np.clip(np.asarray(priors, np.float64), 1e-10, 0.5 - 1e-10)
    return np.log((1 - p) / p).astype(np.float32)


def decode(graph: dict, syndromes: np.ndarray, llr: np.ndarray, *, pre_iter: int, num_sets: int,
           set_max_iter: int, stop_nconv: int, gamma0: float, gamma_legs: Optional[np.ndarray],
           algo: str = "relay", last_leg: bool = False, alpha: Optional[float] = None,
           alpha_scaling: float = 1.0, beta: Optional[float] = None, mix: str = "separate",
           data_type: str = "float32", skip_relay_legs: bool = False,
           llr_per_shot=None, gamma_pre=None, init_posterior=None, gamma_legs_shot=None,
           threads: int = 0) -> dict:
    """Run the oracle on B shots.  Returns errors/weights/weight_fixed/found_count/iterations/last_posterior."""
    syn = _c(syndromes, np.uint8)
    B = syn.shape[0]
    V = graph["V"]
    g = _Graph(graph["C"], graph["V"], graph["E"], _p(graph["chk_ptr"]), _p(graph["edge_var"]),
               _p(graph["var_ptr"]), _p(graph["var_edges"]))
    use_alpha, at = alpha_table(alpha, alpha_scaling, max(pre_iter, set_max_iter))
    prm = _Params(pre_iter, num_sets, set_max_iter, stop_nconv, 1 if last_leg else 0,
                  1 if use_alpha else 0, 1 if beta is not None else 0, float(beta or 0.0),
                  MIX_MODES[mix], MSG_TYPES[data_type], 1 if skip_relay_legs else 0, threads)
    llr = _c(llr, np.float32)
    gl = _c(gamma_legs, np.float32) if gamma_legs is not None else np.zeros((max(num_sets, 1), V), np.float32)
    gp = _c(gamma_pre, np.float32)
    if algo == "plain":
        gamma0, gp = 0.0, None
    ls = _c(llr_per_shot, np.float32)
    ip = _c(init_posterior, np.float32)
    gls = _c(gamma_legs_shot, np.float32)
    inp = _Inputs(B, _p(syn), _p(llr), _p(ls), float(np.float32(gamma0)), _p(gp), _p(gl), _p(gls),
                  0 if gls is None else int(gls.shape[1]), _p(ip), _p(at))
    out = {
        "errors": np.zeros((B, V), np.uint8),
        "weights": np.zeros(B, np.float32),
        "weight_fixed": np.zeros(B, np.int64),
        "found_count": np.zeros(B, np.int32),
        "iterations": np.zeros(B, np.int32),
        "last_posterior": np.zeros((B, V), np.float64),
    }
    o = _Outputs(_p(out["errors"]), _p(out["weights"]), _p(out["weight_fixed"]), _p(out["found_count"]),
                 _p(out["iterations"]), _p(out["last_posterior"]))
    rc = lib().rbo_decode(ct.byref(g), ct.byref(prm), ct.byref(inp), ct.byref(o))
    if rc != 0:
        raise RuntimeError(f"oracle failed with status {rc}")
    out["valid_mask"] = out["found_count"] >= stop_nconv
    return out


def default_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
