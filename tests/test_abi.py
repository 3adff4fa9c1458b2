"""The C ABI library: it loads, exports every symbol include/relaybp.h declares, and
rejects malformed graphs before touching the GPU (CPU only; no compute calls)."""

from __future__ import annotations

import ctypes as ct
import re
from pathlib import Path

import numpy as np
import pytest

from pelagos_b200 import _native as nat

HEADER = Path(__file__).resolve().parent.parent / "include" / "relaybp.h"


def _declared() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"RBP_API\s+[\w\s\*]+?\b(rbp_\w+)\s*\(", text))


def test_library_loads_and_exports_header_symbols():
    lib = nat.lib()
    declared = _declared()
    assert declared == set(nat.EXPORTED_SYMBOLS)
    for name in declared:
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.rbp_version()


def test_library_exports_nothing_else():
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", str(nat.LIB_PATH)], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("nm not available")
    syms = {ln.split()[-1] for ln in out.stdout.splitlines() if " T " in ln}
    assert {s for s in syms if s.startswith("rbp_")} == set(nat.EXPORTED_SYMBOLS)


def _graph_args(chk_ptr, edge_var, var_ptr, var_edges):
    arrs = [np.ascontiguousarray(a, np.int32) for a in (chk_ptr, edge_var, var_ptr, var_edges)]
    return arrs, [nat.i32_ptr(a) for a in arrs]


@pytest.mark.parametrize("case", ["bad_ptr_end", "var_out_of_range", "not_permutation", "nonpositive"])
def test_graph_create_rejects_malformed_input(case):
    lib = nat.lib()
    chk_ptr, edge_var = [0, 2, 4], [0, 1, 1, 2]
    var_ptr, var_edges = [0, 1, 3, 4], [0, 1, 2, 3]
    C, V, E = 2, 3, 4
    if case == "bad_ptr_end":
        chk_ptr = [0, 2, 3]
    elif case == "var_out_of_range":
        edge_var = [0, 1, 1, 7]
    elif case == "not_permutation":
        var_edges = [1, 0, 2, 3]
    elif case == "nonpositive":
        V = 0
    keep, ptrs = _graph_args(chk_ptr, edge_var, var_ptr, var_edges)
    out = ct.c_void_p()
    rc = lib.rbp_graph_create(C, V, E, *ptrs, 0, ct.byref(out))
    assert rc == nat.RBP_ERR_ARGUMENT
    assert lib.rbp_last_error().decode()
    assert not out.value


def test_graph_create_rejects_oversized_layout():
    """A shot's messages must fit the shared-memory layout (padded degree * C < 65535)."""
    lib = nat.lib()
    C, deg = 10000, 7
    V = C * deg
    chk_ptr = np.arange(0, C * deg + 1, deg)
    edge_var = np.arange(V)
    var_ptr = np.arange(V + 1)
    var_edges = np.arange(V)
    keep, ptrs = _graph_args(chk_ptr, edge_var, var_ptr, var_edges)
    out = ct.c_void_p()
    assert lib.rbp_graph_create(C, V, V, *ptrs, 0, ct.byref(out)) == nat.RBP_ERR_UNSUPPORTED


def test_null_arguments():
    lib = nat.lib()
    assert lib.rbp_decode(None, 1, None, None, None) == nat.RBP_ERR_ARGUMENT
    assert lib.rbp_graph_destroy(None) == nat.RBP_OK
    assert lib.rbp_decoder_destroy(None) == nat.RBP_OK
