"""Adapter argument handling that needs no GPU (the reference's RelayDecoder checks,
src/pelagos/adapter.py:96-160)."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.sparse import csr_matrix

import pelagos_b200
from pelagos_b200.adapter import DecodeResult, RelayDecoder

H = csr_matrix(np.array([[1, 1, 0], [0, 1, 1]], np.uint8))


def test_aliases_point_at_the_adapter():
    assert pelagos_b200.RelayDecoderF32 is pelagos_b200.RelayDecoder
    assert pelagos_b200.RelayDecoderF64 is pelagos_b200.RelayDecoder


def test_configs_are_required():
    with pytest.raises(ValueError, match="msl_config and relay_config"):
        RelayDecoder(H, msl_config={"error_priors": np.full(3, 0.1)})
    with pytest.raises(ValueError, match="error_priors"):
        RelayDecoder(H, msl_config={}, relay_config={})


def test_unsupported_data_type_and_execution():
    with pytest.raises(ValueError, match="data_type"):
        RelayDecoder(H, msl_config={"error_priors": np.full(3, 0.1)}, relay_config={}, data_type="int8")
    with pytest.raises(NotImplementedError, match="process"):
        RelayDecoder(H, msl_config={"error_priors": np.full(3, 0.1)}, relay_config={},
                     backend_config={"execution": "process", "data_type": "float32"})


def test_decode_result_defaults():
    r = DecodeResult(decoding=np.zeros(3, np.int8), success=True, iterations=4)
    assert r.decoding_quality == float("inf") and r.found_count is None and not r.converged
