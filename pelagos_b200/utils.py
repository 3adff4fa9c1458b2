"""Host-side numerics utilities with the reference's names and behaviour.

Each function mirrors the function of the same name in the reference's
``src/pelagos/utils.py`` (cited per function) so callers and tests written
against the reference keep working.
"""

from __future__ import annotations

from typing import Optional

import numpy as np
import torch

GAMMA_DRAW_MODES = ("broadcast", "per_row")

#: Priors are clipped into [P_MIN, P_MAX] (utils.py:101, 243).
P_MIN = 1e-10
P_MAX = 0.5 - 1e-10


def compute_log_prior_ratios(error_priors: np.ndarray) -> np.ndarray:
    """log((1 - p) / p) in float64 after clipping p, returned as float32 (utils.py:88-107)."""
    p = np.clip(error_priors, P_MIN, P_MAX)
    return np.log((1 - p) / p).astype(np.float32)


def validate_error_priors(error_priors: np.ndarray) -> np.ndarray:
    """1-D check and clip, printing a warning when clipping changed a value (utils.py:231-251)."""
    error_priors = np.asarray(error_priors)
    if error_priors.ndim != 1:
        raise ValueError("error_priors must be 1D array")
    clipped = np.clip(error_priors, P_MIN, P_MAX)
    if np.any(clipped != error_priors):
        print("Warning: error_priors were clipped to avoid numerical issues")
    return clipped


def validate_csr_matrix(H_csr) -> bool:
    """Sparse, non-empty, at least one nonzero; warn on non-binary data (utils.py:254-272)."""
    from scipy.sparse import csr_matrix, issparse

    if not issparse(H_csr):
        raise ValueError("Input must be a scipy.sparse matrix (any format)")
    if not isinstance(H_csr, csr_matrix):
        H_csr = H_csr.tocsr()
    if H_csr.shape[0] == 0 or H_csr.shape[1] == 0:
        raise ValueError("Matrix cannot be empty")
    if H_csr.nnz == 0:
        raise ValueError("Matrix cannot have zero non-zero elements")
    if not np.all((H_csr.data == 0) | (H_csr.data == 1)):
        print("Warning: Matrix contains non-binary values, will be treated as binary")
    return True


def bitpack_errors(errors: torch.Tensor, bits_per_word: int = 32) -> torch.Tensor:
    """[B, V] 0/1 -> [B, ceil(V/bits_per_word)] int32, bit i of word w = column w*bits+i (utils.py:32-60)."""
    B, V = errors.shape
    words = (V + bits_per_word - 1) // bits_per_word
    padded = torch.zeros(B, words * bits_per_word, dtype=torch.int64, device=errors.device)
    padded[:, :V] = errors.to(torch.int64) & 1
    shifts = torch.arange(bits_per_word, device=errors.device, dtype=torch.int64)
    packed = (padded.view(B, words, bits_per_word) << shifts).sum(dim=2)
    # two's-complement wrap into int32 (bit 31 set -> negative), as a 32-bit OR would give
    packed = torch.where(packed >= 2**31, packed - 2**32, packed)
    return packed.to(torch.int32)


def bitunpack_errors(packed: torch.Tensor, V: int, bits_per_word: int = 32) -> torch.Tensor:
    """Inverse of bitpack_errors (utils.py:63-85)."""
    B, words = packed.shape
    shifts = torch.arange(bits_per_word, device=packed.device, dtype=torch.int64)
    bits = (packed.to(torch.int64).unsqueeze(-1) >> shifts) & 1
    return bits.reshape(B, words * bits_per_word)[:, :V].to(torch.uint8)


def sample_gamma_uniform(rows: int, V: int, gamma_min: float, gamma_max: float, device,
                         seed: Optional[int] = None) -> torch.Tensor:
    """gamma_min + (gamma_max - gamma_min) * U[0,1) from a private generator (utils.py:128-160)."""
    gen = None
    if seed is not None:
        gen = torch.Generator(device=device)
        gen.manual_seed(seed)
    u = torch.rand(rows, V, device=device, generator=gen)
    return gamma_min + (gamma_max - gamma_min) * u


def sample_gamma_scalar(B: int, V: int, gamma_value: float, device) -> torch.Tensor:
    """[B, V] filled with gamma_value (utils.py:163-178)."""
    return torch.full((B, V), gamma_value, device=device)


def sample_gamma_per_variable(rows: int, V: int, gamma_intervals: torch.Tensor, device,
                              seed: Optional[int] = None) -> torch.Tensor:
    """low_v + (high_v - low_v) * U[0,1) per variable (utils.py:181-225)."""
    gen = None
    if seed is not None:
        gen = torch.Generator(device=device)
        gen.manual_seed(seed)
    if gamma_intervals.ndim != 2 or gamma_intervals.shape[0] != V or gamma_intervals.shape[1] != 2:
        raise ValueError(
            f"gamma_intervals must have shape (V={V}, 2), got {tuple(gamma_intervals.shape)}")
    u = torch.rand(rows, V, device=device, generator=gen)
    low = gamma_intervals[:, 0].unsqueeze(0)
    high = gamma_intervals[:, 1].unsqueeze(0)
    return low + (high - low) * u


def alpha_schedule(alpha: Optional[float], scaling: float, n: int) -> tuple[bool, np.ndarray]:
    """Per-iteration normalized min-sum factor, as _run_bp_iteration computes it (decoder.py:2648-2660).

    Returns (use_alpha, table[n] float32).  alpha None -> unused; 0 -> ramp
    1 - 2^(-(t+1)/scaling); otherwise the constant alpha (negative -> 1).
    """
    n = max(int(n), 1)
    if alpha is None:
        return False, np.ones(n, np.float32)
    a = float(alpha)
    if a == 0.0:
        s = float(scaling or 1.0)
        return True, np.array([1.0 - (2.0 ** (-((t + 1) / s))) for t in range(n)], dtype=np.float32)
    if a < 0.0:
        return True, np.ones(n, np.float32)
    return True, np.full(n, a, dtype=np.float32)
