"""ctypes binding of the C ABI in include/relaybp.h (librelaybp.so).

The shared library is built in-tree (``pelagos_b200/_lib/librelaybp.so``) by
``pelagos_b200.build``.  There is no fallback: if the library is missing or
fails to load, every decoder entry point raises ``NativeLibraryError``.
"""

from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

LIB_DIR = Path(__file__).resolve().parent / "_lib"
LIB_PATH = LIB_DIR / "librelaybp.so"

RBP_OK = 0
RBP_ERR_ARGUMENT = 1
RBP_ERR_CUDA = 2
RBP_ERR_UNSUPPORTED = 3

RBP_MSG_F32 = 0
RBP_MSG_F16 = 1
RBP_MSG_BF16 = 2
RBP_MSG_F64 = 3

RBP_MIX_SEPARATE = 0
RBP_MIX_FMA_GP = 1
RBP_MIX_FMA_LP = 2

RBP_LAUNCH_ALL = 0
RBP_LAUNCH_PRE = 1
RBP_LAUNCH_LEGS = 2

#: Every symbol include/relaybp.h declares.
EXPORTED_SYMBOLS = (
    "rbp_last_error",
    "rbp_version",
    "rbp_graph_create",
    "rbp_graph_destroy",
    "rbp_decoder_create",
    "rbp_decoder_destroy",
    "rbp_decoder_set_llr",
    "rbp_decoder_configure",
    "rbp_decoder_query",
    "rbp_decoder_configure_kind",
    "rbp_decoder_query_kind",
    "rbp_state_bytes",
    "rbp_state_posterior_offset",
    "rbp_decode",
    "rbp_decode_static",
    "rbp_mixed_create",
    "rbp_mixed_destroy",
    "rbp_mixed_decode",
    "rbp_mixed_capture",
    "rbp_mixed_replay",
    "rbp_mixed_query",
    "rbp_mixed_configure",
    "rbp_net_param_count",
    "rbp_net_create",
    "rbp_net_destroy",
    "rbp_net_set_params",
    "rbp_net_get_params",
    "rbp_net_forward",
    "rbp_net_train_step",
    "rbp_net_propose",
    "rbp_gf2_matvec",
)

#: Bytes of the static scratch array rbp_decode_static uses (RBP_STATIC_SCRATCH_BYTES).
STATIC_SCRATCH_BYTES = 1 << 20


class NativeLibraryError(RuntimeError):
    """The CUDA library is missing or a native call failed."""


class RbpParams(ct.Structure):
    _fields_ = [
        ("pre_iter", ct.c_int32),
        ("num_sets", ct.c_int32),
        ("set_max_iter", ct.c_int32),
        ("stop_nconv", ct.c_int32),
        ("msg_type", ct.c_int32),
        ("last_leg", ct.c_int32),
        ("use_alpha", ct.c_int32),
        ("use_beta", ct.c_int32),
        ("beta", ct.c_float),
        ("mix_mode", ct.c_int32),
    ]


class _Sized(ct.Structure):
    """A struct whose first field, struct_size, carries sizeof(struct): filled in on construction,
    so the library can reject a caller whose declaration differs from include/relaybp.h."""

    def __init__(self, *args, **kw):
        super().__init__(*args, **kw)
        if "struct_size" not in kw:
            self.struct_size = ct.sizeof(self)


class RbpBatch(_Sized):
    _fields_ = [
        ("struct_size", ct.c_uint32),
        ("syndromes", ct.c_void_p),
        ("llr_per_shot", ct.c_void_p),
        ("gamma_pre", ct.c_void_p),
        ("gamma0", ct.c_float),
        ("init_posterior", ct.c_void_p),
        ("gamma_legs_shot", ct.c_void_p),
        ("n_shot_legs", ct.c_int32),
        ("pre_iter", ct.c_int32),
        ("skip_relay_legs", ct.c_int32),
        ("resume_state", ct.c_void_p),
        ("suspend_state", ct.c_void_p),
        ("legs_begin", ct.c_int32),
        ("legs_end", ct.c_int32),
        ("shot_leg_rows", ct.c_int32),
        ("shot_order", ct.c_void_p),
        ("queue_len", ct.c_void_p),
        ("solved_gamma", ct.c_float),
        ("solved_legs", ct.c_int32),
        ("suspend_unsolved", ct.c_int32),
        ("parity_first", ct.c_int32),
    ]


class RbpNetHparams(ct.Structure):
    _fields_ = [
        ("lr", ct.c_float),
        ("beta1", ct.c_float),
        ("beta2", ct.c_float),
        ("eps", ct.c_float),
        ("weight_decay", ct.c_float),
        ("w_neg", ct.c_float),
    ]


class RbpOutputs(_Sized):
    _fields_ = [
        ("struct_size", ct.c_uint32),
        ("errors", ct.c_void_p),
        ("errors_packed", ct.c_void_p),
        ("weights", ct.c_void_p),
        ("weight_fixed", ct.c_void_p),
        ("found_count", ct.c_void_p),
        ("iterations", ct.c_void_p),
        ("last_posterior", ct.c_void_p),
    ]


_lib = None


def _declare(lib):
    P = ct.c_void_p
    i32, i64 = ct.c_int32, ct.c_int64
    i32p = ct.POINTER(ct.c_int32)
    f32p = ct.POINTER(ct.c_float)
    lib.rbp_last_error.restype = ct.c_char_p
    lib.rbp_last_error.argtypes = []
    lib.rbp_version.restype = ct.c_char_p
    lib.rbp_version.argtypes = []
    lib.rbp_graph_create.restype = ct.c_int
    lib.rbp_graph_create.argtypes = [i32, i32, i32, i32p, i32p, i32p, i32p, i32, ct.POINTER(P)]
    lib.rbp_graph_destroy.restype = ct.c_int
    lib.rbp_graph_destroy.argtypes = [P]
    lib.rbp_decoder_create.restype = ct.c_int
    lib.rbp_decoder_create.argtypes = [P, ct.POINTER(RbpParams), f32p, f32p, f32p, i32, ct.POINTER(P)]
    lib.rbp_decoder_destroy.restype = ct.c_int
    lib.rbp_decoder_destroy.argtypes = [P]
    lib.rbp_decoder_set_llr.restype = ct.c_int
    lib.rbp_decoder_set_llr.argtypes = [P, f32p]
    lib.rbp_decoder_configure.restype = ct.c_int
    lib.rbp_decoder_configure.argtypes = [P, i32, i32, i32]
    lib.rbp_decoder_query.restype = ct.c_int
    lib.rbp_decoder_query.argtypes = [P, ct.POINTER(i64), ct.POINTER(i64), i32p, i32p, i32p, i32p]
    lib.rbp_decoder_configure_kind.restype = ct.c_int
    lib.rbp_decoder_configure_kind.argtypes = [P, i32, i32, i32, i32, i32]
    lib.rbp_decoder_query_kind.restype = ct.c_int
    lib.rbp_decoder_query_kind.argtypes = [P, i32, i32p, i32p, i32p, i32p, i32p]
    lib.rbp_state_bytes.restype = ct.c_int
    lib.rbp_state_bytes.argtypes = [P, ct.POINTER(i64)]
    lib.rbp_state_posterior_offset.restype = ct.c_int
    lib.rbp_state_posterior_offset.argtypes = [P, ct.POINTER(i64)]
    lib.rbp_decode.restype = ct.c_int
    lib.rbp_decode.argtypes = [P, i64, ct.POINTER(RbpBatch), ct.POINTER(RbpOutputs), P]
    lib.rbp_decode_static.restype = ct.c_int
    lib.rbp_decode_static.argtypes = [i32, i32, i32, i32p, i32p, i32p, i32p, ct.POINTER(RbpParams), P, P, P, i32,
                                      i32, i64, ct.POINTER(RbpBatch), ct.POINTER(RbpOutputs), P]
    lib.rbp_mixed_create.restype = ct.c_int
    lib.rbp_mixed_create.argtypes = [ct.POINTER(P), i32, ct.POINTER(P)]
    lib.rbp_mixed_destroy.restype = ct.c_int
    lib.rbp_mixed_destroy.argtypes = [P]
    for f in (lib.rbp_mixed_decode,):
        f.restype = ct.c_int
        f.argtypes = [P, ct.POINTER(i64), ct.POINTER(RbpBatch), ct.POINTER(RbpOutputs), P]
    lib.rbp_mixed_capture.restype = ct.c_int
    lib.rbp_mixed_capture.argtypes = [P, ct.POINTER(i64), ct.POINTER(RbpBatch), ct.POINTER(RbpOutputs)]
    lib.rbp_mixed_replay.restype = ct.c_int
    lib.rbp_mixed_replay.argtypes = [P, P]
    lib.rbp_mixed_query.restype = ct.c_int
    lib.rbp_mixed_query.argtypes = [P, i32, i32p, i32p, i32p, i32p]
    lib.rbp_mixed_configure.restype = ct.c_int
    lib.rbp_mixed_configure.argtypes = [P, ct.POINTER(i32)]
    lib.rbp_net_param_count.restype = ct.c_int
    lib.rbp_net_param_count.argtypes = [ct.POINTER(i64)]
    lib.rbp_net_create.restype = ct.c_int
    lib.rbp_net_create.argtypes = [P, f32p, ct.POINTER(P)]
    lib.rbp_net_destroy.restype = ct.c_int
    lib.rbp_net_destroy.argtypes = [P]
    for f in (lib.rbp_net_set_params, lib.rbp_net_get_params):
        f.restype = ct.c_int
        f.argtypes = [P, P, P]
    lib.rbp_net_forward.restype = ct.c_int
    lib.rbp_net_forward.argtypes = [P, i64, P, P, P, P]
    lib.rbp_net_train_step.restype = ct.c_int
    lib.rbp_net_train_step.argtypes = [P, i64, P, P, P, ct.POINTER(RbpNetHparams), P, P, P]
    lib.rbp_net_propose.restype = ct.c_int
    lib.rbp_net_propose.argtypes = [P, i64, P, P, i64, ct.c_float, ct.c_float, P, P, P, P, P]
    lib.rbp_gf2_matvec.restype = ct.c_int
    lib.rbp_gf2_matvec.argtypes = [P, i64, i32, P, P, i32, P, P]
    return lib


def lib():
    """Load (once) and return the native library; raise if it is not built."""
    global _lib
    if _lib is None:
        path = Path(os.environ.get("PELAGOS_B200_LIB", LIB_PATH))
        if not path.exists():
            raise NativeLibraryError(
                f"CUDA library {path} is not built; run `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `python -m pelagos_b200.build`")
        try:
            _lib = _declare(ct.CDLL(str(path)))
        except OSError as exc:  # pragma: no cover - depends on the host
            raise NativeLibraryError(f"cannot load {path}: {exc}") from exc
    return _lib


def check(rc: int, what: str) -> None:
    if rc != RBP_OK:
        msg = lib().rbp_last_error().decode(errors="replace")
        kind = {RBP_ERR_ARGUMENT: ValueError, RBP_ERR_UNSUPPORTED: NotImplementedError}.get(rc)
        if kind is not None:
            raise kind(f"{what}: {msg}")
        raise NativeLibraryError(f"{what} failed (status {rc}): {msg}")


def f32_ptr(arr):
    return arr.ctypes.data_as(ct.POINTER(ct.c_float)) if arr is not None else None


def i32_ptr(arr):
    return arr.ctypes.data_as(ct.POINTER(ct.c_int32))
