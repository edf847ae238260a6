"""Synthetic cls5 workloads: Stage-1 unit streams and seeded planted targets.

Units are generated by the reference's Stage-1 rule (fourcore_hunt_v3.cpp:
371-381 over fourcore_classes_v3.hpp:137-154) through the engine's own
``s615_unit_candidates``; the emitted lines have the ``.buc`` format
``cls B u``.  Plants follow the reference's plant shape (solve_516_v3.cu:
1149-1170): base = (14e)^6 + (21d)^6 + 42^6 (c1^6 + c2^6), one residue per axis
and fmax equal to the planted value, so the planted point is on the grid.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

import s615

M42 = 42**6


def eligible(B: int) -> bool:
    return B > 1 and math.gcd(B, 42) == 1


def cls5_units(lo: int, hi: int) -> List[Tuple[int, int]]:
    """All Stage-1 cls5 units (B, u) with B in [lo, hi], gcd(B,42)=1."""
    out = []
    for B in range(lo, hi + 1):
        if not eligible(B):
            continue
        for u in s615.unit_candidates(B, 5):
            out.append((B, u))
    return out


def write_buc(path: str, units: List[Tuple[int, int]], cls: int = 5) -> None:
    with open(path, "w") as f:
        for B, u in units:
            f.write(f"{cls} {B} {u}\n")


@dataclass
class Plant:
    B: int
    u: int
    e: int   # x14 term
    d: int   # x21 term
    c1: int
    c2: int

    @property
    def base(self) -> int:
        return (14 * self.e) ** 6 + (21 * self.d) ** 6 + M42 * (self.c1**6 + self.c2**6)

    @property
    def T(self) -> int:
        return self.c1**6 + self.c2**6

    @property
    def fp(self) -> int:
        return self.T % 2**64


def plants(n: int, seed: int, B_lo: int, B_hi: int, N: int) -> List[Plant]:
    """n planted targets with B uniform over the eligible band, e <= (B-1)/14,
    d <= (B-1)/21, c1 != c2 in [1, N], u a multiple of 6 below B."""
    rng = np.random.RandomState(seed)
    out = []
    while len(out) < n:
        B = int(rng.randint(B_lo, B_hi + 1))
        if not eligible(B):
            continue
        e = int(rng.randint(1, (B - 1) // 14 + 1))
        d = int(rng.randint(1, (B - 1) // 21 + 1))
        c1 = int(rng.randint(1, N + 1))
        c2 = int(rng.randint(1, N + 1))
        if c1 == c2:
            continue
        u = 6 * int(rng.randint(1, max(2, (B - 1) // 6)))
        out.append(Plant(B, u, e, d, min(c1, c2), max(c1, c2)))
    return out


def plant_unit(p: Plant, N: int) -> "s615.Unit":
    return s615.make_plant(p.base, p.e, p.d, lim=N, u=p.u, B=p.B)


def unit_array(units: List[Tuple[int, int]], plant_list: List[Plant], N: int):
    """One s615_unit array: Stage-1 units first, then plants."""
    n = len(units) + len(plant_list)
    arr = (s615.Unit * max(n, 1))()
    for i, (B, u) in enumerate(units):
        arr[i].cls, arr[i].kind, arr[i].B, arr[i].u = 5, 0, B, u
    for j, p in enumerate(plant_list):
        arr[len(units) + j] = plant_unit(p, N)
    return arr, n
