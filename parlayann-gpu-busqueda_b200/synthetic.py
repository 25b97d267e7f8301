"""Seeded synthetic vector sets with the shapes of the reference's benchmark data.

The reference runs on MSSPACEV-1M (1,000,000 int8 vectors, d=100, 29,316 queries;
reference README.md:52-53), which is not available here. These generators stand in for
it: Gaussian mixtures rounded and clipped to 8 bits. PRNG: numpy PCG64 seeded with
``seed``; centres, base points and queries use independent child streams, so the base
does not depend on the number of queries.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class MixtureLaw:
    dim: int
    n_centers: int
    center_lo: float
    center_hi: float
    sigma: float
    zero_frac: float      # fraction of coordinates forced to exactly 0
    signed: bool          # int8 (True) or uint8

    def _clip(self, x: np.ndarray) -> np.ndarray:
        lo, hi = (-128, 127) if self.signed else (0, 255)
        return np.clip(np.rint(x), lo, hi).astype(np.int8 if self.signed else np.uint8)

    def sample(self, n: int, seed: int, stream: int, chunk: int = 1 << 20) -> np.ndarray:
        """stream 0: base points; 1: queries; s >= 2: further independent query sets."""
        ss = np.random.SeedSequence(seed)
        c_seq, b_seq, q_seq = ss.spawn(3)
        centers = np.random.Generator(np.random.PCG64(c_seq)).uniform(
            self.center_lo, self.center_hi, size=(self.n_centers, self.dim)).astype(np.float32)
        if stream == 0:
            seq = b_seq
        elif stream == 1:
            seq = q_seq
        else:
            seq = np.random.SeedSequence(seed, spawn_key=(1000 + stream,))
        rng = np.random.Generator(np.random.PCG64(seq))
        out = np.empty((n, self.dim), dtype=np.int8 if self.signed else np.uint8)
        for s in range(0, n, chunk):
            e = min(n, s + chunk)
            lab = rng.integers(0, self.n_centers, size=e - s)
            x = centers[lab] + rng.standard_normal((e - s, self.dim), dtype=np.float32) * self.sigma
            if self.zero_frac > 0:
                x[rng.random((e - s, self.dim), dtype=np.float32) < self.zero_frac] = 0.0
            out[s:e] = self._clip(x)
        return out


# mixture laws of the workloads: C1 10k int8 d=100 (64 centres); C2-C3-C5 1M int8 d=100 (1,024 centres); C4 10M uint8 d=128 (4,096 centres)
LAW_C1 = MixtureLaw(dim=100, n_centers=64, center_lo=-40, center_hi=40, sigma=12,
                    zero_frac=0.0, signed=True)
LAW_C2 = MixtureLaw(dim=100, n_centers=1024, center_lo=-40, center_hi=40, sigma=10,
                    zero_frac=0.30, signed=True)
LAW_C4 = MixtureLaw(dim=128, n_centers=4096, center_lo=24, center_hi=232, sigma=20,
                    zero_frac=0.40, signed=False)


def dataset(law: MixtureLaw, n: int, nq: int, seed: int = 0):
    """(base[n, dim], queries[nq, dim]) drawn from the same law."""
    return law.sample(n, seed, 0), law.sample(nq, seed, 1)


def c1(seed: int = 0):
    return dataset(LAW_C1, 10_000, 1_000, seed)


def c2(seed: int = 0, n: int = 1_000_000, nq: int = 29_316):
    return dataset(LAW_C2, n, nq, seed)


def c4(seed: int = 0, n: int = 10_000_000, nq: int = 100_000):
    return dataset(LAW_C4, n, nq, seed)


# 18 beam widths of the full-shape sweep: round(10 * 50**(i/17))
LS_SWEEP = [int(round(10 * 50 ** (i / 17))) for i in range(18)]
