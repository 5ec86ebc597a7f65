"""Seeded synthetic workloads of the benchmark configurations.

Inputs are synthetic: base scalars come from seeds ``LE32(i)`` and prefixes
from splitmix64 seeded by the configuration number, symbols ``next() % 32``
over the base32 alphabet and lengths ``lo + next() % (hi - lo + 1)``.

    config 1  4096 lanes x 256 chain steps (2^20 candidates), one 4-char prefix
    config 2  2^32 candidates, one 6-char prefix
    config 3  2^32 candidates, 10,000 prefixes of 3..8 chars
    config 4  64 searches, 1..5,000 prefixes (log-uniform) of 4..7 chars, quota 1..16
    config 5  2,000 requests, Poisson arrivals at 50/s, 1..200 prefixes of 4..7, quota 1..16
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

ALPHABET = "abcdefghijklmnopqrstuvwxyz234567"
MASK = (1 << 64) - 1


class SplitMix64:
    """The splitmix64 generator (Steele, Lea, Flood 2014)."""

    def __init__(self, seed: int):
        self.state = seed & MASK

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        """A double in [0, 1) from the top 53 bits."""
        return (self.next() >> 11) * (1.0 / (1 << 53))

    def prefix(self, lo: int, hi: int) -> str:
        n = lo + self.next() % (hi - lo + 1)
        return "".join(ALPHABET[self.next() % 32] for _ in range(n))


def seed(i: int) -> bytes:
    return int(i).to_bytes(32, "little")


def log_uniform_count(rng: SplitMix64, hi: int) -> int:
    """floor(exp(u ln hi)), u uniform in [0, 1): 1..hi-1, log-uniform."""
    return max(1, int(math.floor(math.exp(rng.uniform() * math.log(hi)))))


@dataclass
class Search:
    index: int
    seed: bytes
    prefixes: list
    quota: int
    arrival: float = 0.0

    def match_probability(self) -> float:
        """Chance one candidate matches some prefix (distinct prefixes, none absorbing another)."""
        uniq = sorted(set(self.prefixes))
        kept = []
        for p in uniq:
            if kept and p.startswith(kept[-1]):
                continue
            kept.append(p)
        return min(1.0, sum(32.0 ** -len(p) for p in kept))

    def expected_candidates(self) -> float:
        return self.quota / self.match_probability()


def config1_prefix() -> str:
    return SplitMix64(1).prefix(4, 4)


def config2_prefix() -> str:
    return SplitMix64(2).prefix(6, 6)


def config3_prefixes(n: int = 10_000):
    r = SplitMix64(3)
    return [r.prefix(3, 8) for _ in range(n)]


def config4_searches(n: int = 64):
    r = SplitMix64(4)
    out = []
    for j in range(n):
        count = log_uniform_count(r, 5000)
        prefixes = [r.prefix(4, 7) for _ in range(count)]
        quota = 1 + r.next() % 16
        out.append(Search(j, seed(j), prefixes, quota))
    return out


def config5_requests(n: int = 2000, rate: float = 50.0):
    r = SplitMix64(5)
    out = []
    t = 0.0
    for j in range(n):
        t += -math.log(1.0 - r.uniform()) / rate
        count = log_uniform_count(r, 200)
        prefixes = [r.prefix(4, 7) for _ in range(count)]
        quota = 1 + r.next() % 16
        out.append(Search(j, seed(j), prefixes, quota, arrival=t))
    return out


def suffix_filters(n: int = 16, length: int = 9):
    """A suffix workload: `n` suffixes of `length` symbols from splitmix64(6),
    each ending in a reachable v3 tail (a symbol of "aiqy", then "d")."""
    rng = SplitMix64(6)
    out = []
    for _ in range(n):
        body = "".join(ALPHABET[rng.next() % 32] for _ in range(length - 2))
        out.append("suffix:" + body + "aiqy"[rng.next() % 4] + "d")
    return out
