"""The C structs of include/relaybp.h against their two Python declarations: the
package's ctypes binding (pelagos_b200/_native.py) and the binding INTEGRATION.md
tells a reference maintainer to add.  A field missing, added or out of order in
either would make rbp_decode read the caller's struct at the wrong offsets.
Also: the library's struct_size check and the allocation-free entry point's
graph validation, both of which reject before any GPU call (CPU only)."""

from __future__ import annotations

import ast
import ctypes as ct
import re
from pathlib import Path

import numpy as np

from pelagos_b200 import _native as nat

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "relaybp.h"
INTEGRATION = ROOT / "INTEGRATION.md"

# header struct name -> (ctypes class in _native, class name in the INTEGRATION.md stub)
STRUCTS = {
    "rbp_params": ("RbpParams", "_Params"),
    "rbp_batch": ("RbpBatch", "_Batch"),
    "rbp_outputs": ("RbpOutputs", "_Outputs"),
    "rbp_net_hparams": ("RbpNetHparams", "_NetHparams"),
}


def _kind_c(ctype: str) -> str:
    ctype = ctype.strip()
    if "*" in ctype:
        return "ptr"
    return {"int32_t": "i32", "uint32_t": "u32", "float": "f32", "int64_t": "i64"}[ctype.replace("const ", "")]


def header_structs() -> dict[str, list[tuple[str, str]]]:
    """typedef struct { ... } name; blocks of the header as [(field, kind)]."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    out = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            parts = [p.strip() for p in decl.split(",")]
            first = re.match(r"(.*?)(\w+)$", parts[0], flags=re.S)
            ctype = first.group(1)
            # "float lr, beta1" declares several fields of one type
            for name_ in [first.group(2)] + parts[1:]:
                fields.append((name_, _kind_c(ctype)))
        out[name] = fields
    return out


def _kind_ctypes(t) -> str:
    if t is ct.c_void_p or issubclass(t, ct._Pointer):
        return "ptr"
    return {ct.c_int32: "i32", ct.c_uint32: "u32", ct.c_float: "f32", ct.c_int64: "i64"}[t]


def _kind_stub(expr: str) -> str:
    return {"P": "ptr", "I32": "i32", "I64": "i64", "ct.c_float": "f32", "ct.c_uint32": "u32",
            "ct.c_int32": "i32", "ct.c_void_p": "ptr"}[expr]


def integration_structs() -> dict[str, list[tuple[str, str]]]:
    """_fields_ of every ctypes class in INTEGRATION.md's python code blocks."""
    out = {}
    for block in re.findall(r"```python\n(.*?)```", INTEGRATION.read_text(), flags=re.S):
        for node in ast.walk(ast.parse(block)):
            if not isinstance(node, ast.ClassDef):
                continue
            for stmt in node.body:
                if isinstance(stmt, ast.Assign) and any(getattr(t, "id", "") == "_fields_" for t in stmt.targets):
                    out[node.name] = [(e.elts[0].value, _kind_stub(ast.unparse(e.elts[1]))) for e in stmt.value.elts]
    return out


def test_header_structs_parsed():
    hs = header_structs()
    assert set(STRUCTS) <= set(hs)
    assert hs["rbp_batch"][0] == ("struct_size", "u32")
    assert hs["rbp_outputs"][0] == ("struct_size", "u32")
    assert len(hs["rbp_batch"]) == 21 and len(hs["rbp_outputs"]) == 8


def test_native_binding_matches_header_field_for_field():
    hs = header_structs()
    for cname, (pyname, _) in STRUCTS.items():
        cls = getattr(nat, pyname)
        got = [(n, _kind_ctypes(t)) for n, t in cls._fields_]
        assert got == hs[cname], cname


def test_integration_stub_matches_header_field_for_field():
    hs, stub = header_structs(), integration_structs()
    for cname, (_, stubname) in STRUCTS.items():
        assert stubname in stub, f"INTEGRATION.md declares no {stubname} for {cname}"
        assert stub[stubname] == hs[cname], cname


def test_struct_size_filled_in():
    assert nat.RbpBatch().struct_size == ct.sizeof(nat.RbpBatch)
    assert nat.RbpOutputs().struct_size == ct.sizeof(nat.RbpOutputs)
    assert nat.RbpBatch(struct_size=3).struct_size == 3


def _static_call(batch, outs, var_edges=(0, 1, 2, 3)):
    """rbp_decode_static on a 2x3 graph with host-side arguments only: every failure path
    exercised here returns before the library selects a device."""
    chk_ptr = np.array([0, 2, 4], np.int32)
    edge_var = np.array([0, 1, 1, 2], np.int32)
    var_ptr = np.array([0, 1, 3, 4], np.int32)
    var_edges = np.array(var_edges, np.int32)
    params = nat.RbpParams(pre_iter=2, num_sets=0, set_max_iter=1, stop_nconv=1, msg_type=nat.RBP_MSG_F32)
    dummy = ct.c_void_p(0x1000)  # never dereferenced on these paths
    return nat.lib().rbp_decode_static(2, 3, 4, nat.i32_ptr(chk_ptr), nat.i32_ptr(edge_var), nat.i32_ptr(var_ptr),
                                       nat.i32_ptr(var_edges), ct.byref(params), dummy, None, None, 0, 0, 4,
                                       ct.byref(batch), ct.byref(outs), None)


def _io():
    d = ct.c_void_p(0x1000)
    return nat.RbpBatch(syndromes=d, pre_iter=2), nat.RbpOutputs(found_count=d, iterations=d)


def test_struct_size_mismatch_rejected():
    batch, outs = _io()
    batch.struct_size = ct.sizeof(nat.RbpBatch) - 8  # a binding with one pointer field fewer
    assert _static_call(batch, outs) == nat.RBP_ERR_ARGUMENT
    assert "struct_size" in nat.lib().rbp_last_error().decode()
    batch, outs = _io()
    outs.struct_size = 0
    assert _static_call(batch, outs) == nat.RBP_ERR_ARGUMENT
    assert "rbp_outputs.struct_size" in nat.lib().rbp_last_error().decode()


def test_static_entry_rejects_duplicated_edges():
    """var_edges listing edge 1 twice (and edge 2 never) is not a permutation: rbp_graph_create
    rejects that graph, and so does the allocation-free entry point."""
    batch, outs = _io()
    assert _static_call(batch, outs, var_edges=(0, 1, 1, 3)) == nat.RBP_ERR_ARGUMENT
    assert "permutation" in nat.lib().rbp_last_error().decode()
