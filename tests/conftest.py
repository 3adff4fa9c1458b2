"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built sm_100a library")


def golden_cases() -> list[str]:
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


class Golden:
    """One fixture written by tests/golden/make_golden.py from the reference decoder."""

    def __init__(self, name: str):
        z = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
        self.name = name
        self.z = {k: z[k] for k in z.files}
        meta = json.loads(str(self.z["meta"]))
        self.kw = meta["kwargs"]
        self.dkw = meta["decode_kwargs"]
        C, V = (int(x) for x in self.z["shape"])
        self.C, self.V = C, V
        from scipy.sparse import csr_matrix

        self.H = csr_matrix((np.ones(self.z["indices"].size, np.uint8), self.z["indices"], self.z["indptr"]),
                            shape=(C, V))
        self.priors = self.z["priors"]
        self.syndromes = self.z["syndromes"]
        self.num_sets = int(self.kw.get("num_sets", 100))

    def arr(self, key):
        return self.z.get(key)

    @property
    def graph(self) -> dict:
        z = self.z
        return {"C": self.C, "V": self.V, "E": int(z["indices"].size), "chk_ptr": z["indptr"],
                "edge_var": z["ref_edge_var"], "var_ptr": z["ref_var_ptr"], "var_edges": z["ref_var_edges"]}

    def leg_table(self) -> np.ndarray:
        """[num_sets, V] gammas the reference's legs used.  Legs the reference never
        reached (every shot had stopped) are NaN; no shot may read them."""
        R, V = self.num_sets, self.V
        t = np.full((max(R, 1), V), np.nan, np.float32)
        if "kw_explicit_gammas" in self.z:
            eg = self.z["kw_explicit_gammas"].astype(np.float32)
            K = eg.shape[0]
            for leg in range(R):
                t[leg] = eg[(leg + 1) % K]
        else:
            d = self.z["leg_draws"]
            t[: d.shape[0]] = d
        return t[:R] if R else np.zeros((0, V), np.float32)

    def decode_args(self) -> dict:
        kw, dkw = self.kw, self.dkw
        return dict(
            pre_iter=int(dkw.get("pre_iter_override", kw.get("pre_iter", 80))),
            num_sets=self.num_sets,
            set_max_iter=int(kw.get("set_max_iter", 60)),
            stop_nconv=int(kw.get("stop_nconv", 5)),
            gamma0=float(kw.get("gamma0", 0.65)),
            algo=kw.get("algo"),
            last_leg=kw.get("unconverged_correction") == "last_leg",
            alpha=kw.get("normalized_min_sum_alpha"),
            alpha_scaling=float(kw.get("alpha_iteration_scaling_factor", 1.0) or 1.0),
            beta=kw.get("offset_min_sum_beta"),
            data_type=kw.get("data_type", "float32"),
            skip_relay_legs=bool(dkw.get("skip_relay_legs", False)),
            llr_per_shot=self.z.get("dkw_prior_llr"),
            gamma_pre=self.z.get("dkw_init_gamma"),
            init_posterior=self.z.get("dkw_init_posterior"),
        )


@pytest.fixture(params=golden_cases())
def golden(request) -> Golden:
    return Golden(request.param)
