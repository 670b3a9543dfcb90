"""Seeded synthetic tables for the benchmark and the parity tests.

No public dataset is involved; every column is drawn with numpy's PCG64 from a
seed fixed per (workload, column), with the shapes and distributions of the
reference's headline configurations:

* table ``t`` (filter / group-by / scan / top-k): ``id`` int64 = 0..N-1;
  ``dept`` text drawn uniformly from 12 labels 'd00'..'d11' (dictionary codes
  into one sorted dictionary); ``score`` float64 uniform [0,100); ``salary``
  int64 uniform [30000, 200000].
* join: build side ``b`` (``key`` = a seeded permutation of 0..B-1, ``payload``
  int64 uniform [0, 1e6)); probe side ``p`` (``key`` int64 uniform [0, 2B),
  ``value`` float64 uniform [0,1)).
* high-cardinality GROUP BY ``g``: ``key`` = pi(r-1) with r ~ Zipf(s=1.1) over
  1..D (D = 10M at full size) and pi a seeded permutation; ``v`` float64
  uniform [0,1).  Zipf draws use rejection-inversion (Hörmann & Derflinger,
  "Rejection-inversion to generate variates from monotone discrete
  distributions", ACM TOMACS 1996), vectorised.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np

from . import Utf8

DEPTS = [f"d{i:02d}" for i in range(12)]


def _rng(*key: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence(list(key))))


def table_t(n: int, seed: int = 1) -> Dict[str, object]:
    """Columns of table t (id, dept, score, salary) with n rows."""
    return {
        "id": np.arange(n, dtype=np.int64),
        "dept": Utf8(_rng(seed, 2).integers(0, 12, size=n, dtype=np.uint32), DEPTS),
        "score": _rng(seed, 3).random(n) * 100.0,
        "salary": _rng(seed, 4).integers(30_000, 200_001, size=n, dtype=np.int64),
    }


def join_tables(n_build: int, n_probe: int, seed: int = 7) -> Tuple[Dict[str, np.ndarray], Dict[str, np.ndarray]]:
    """(build, probe) columns: build key a permutation of 0..n_build-1, probe
    keys uniform over [0, 2*n_build) so about half of them match."""
    build = {
        "key": _rng(seed, 1).permutation(n_build).astype(np.int64),
        "payload": _rng(seed, 2).integers(0, 1_000_000, size=n_build, dtype=np.int64),
    }
    probe = {
        "key": _rng(seed, 3).integers(0, 2 * n_build, size=n_probe, dtype=np.int64),
        "value": _rng(seed, 4).random(n_probe),
    }
    return build, probe


def zipf(n: int, s: float, domain: int, rng: np.random.Generator) -> np.ndarray:
    """n draws from Zipf(s) over 1..domain (P(k) ~ k^-s), rejection-inversion."""
    one_m_s = 1.0 - s

    def H(x):  # integral of x^-s, shifted so H(1) = 0
        return np.expm1(one_m_s * np.log(x)) / one_m_s

    def H_inv(y):
        return np.exp(np.log1p(y * one_m_s) / one_m_s)

    h_x1 = float(H(np.float64(1.5))) - 1.0
    h_n = float(H(np.float64(domain + 0.5)))
    s_cut = 2.0 - float(H_inv(H(np.float64(2.5)) - 2.0 ** -s))
    out = np.empty(n, dtype=np.int64)
    filled = 0
    while filled < n:
        m = int((n - filled) * 1.1) + 1024
        u = h_n + rng.random(m) * (h_x1 - h_n)
        x = H_inv(u)
        k = np.clip(np.floor(x + 0.5), 1, domain)
        ok = (k - x <= s_cut) | (u >= H(k + 0.5) - np.exp(-s * np.log(k)))
        acc = k[ok].astype(np.int64)
        take = min(len(acc), n - filled)
        out[filled:filled + take] = acc[:take]
        filled += take
    return out


def groupby_table(n: int, distinct: int = 10_000_000, s: float = 1.1, seed: int = 11) -> Dict[str, np.ndarray]:
    """Columns key (Zipf over `distinct` values, permuted) and v."""
    r = zipf(n, s, distinct, _rng(seed, 1))
    perm = _rng(seed, 2).permutation(distinct).astype(np.int64)
    return {"key": perm[r - 1], "v": _rng(seed, 3).random(n)}


def zipf_pmf(s: float, domain: int) -> np.ndarray:
    k = np.arange(1, domain + 1, dtype=np.float64)
    w = k ** -s
    return w / w.sum()
