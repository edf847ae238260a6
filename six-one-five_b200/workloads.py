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


# ------------------------------------------------- mixed-class unit streams
MIX = {2: 0.04, 3: 0.01, 4: 0.48, 5: 0.47}   # class shares of the mixed stream
FREE = {2: 14, 3: 21, 4: 7}                    # free factor of classes 2-4
FREE_MOD = {2: 729, 3: 64, 4: 46656}


def mixed_units(n: int, seed: int, B_lo: int, B_hi: int, log_uniform: bool = True,
                mix=MIX) -> List[Tuple[int, int, int]]:
    """n Stage-1 units (cls, B, u): B log-uniform (or uniform) on [B_lo, B_hi]
    with gcd(B, 42) = 1, the class drawn by `mix`, u uniform among that B's
    units of the class (fourcore_classes_v3.hpp:137-154)."""
    rng = np.random.RandomState(seed)
    classes = sorted(mix)
    p = np.array([mix[c] for c in classes], dtype=float)
    p /= p.sum()
    out = []
    while len(out) < n:
        if log_uniform:
            B = int(math.exp(rng.uniform(math.log(B_lo), math.log(B_hi))))
        else:
            B = int(rng.randint(B_lo, B_hi + 1))
        if not eligible(B):
            continue
        c = int(classes[rng.choice(len(classes), p=p)])
        us = s615.unit_candidates(B, c)
        if not us:
            continue
        out.append((c, B, int(us[rng.randint(len(us))])))
    return out


def plants234(n: int, seed: int, B_lo: int, B_hi: int, N: int):
    """Planted class 2-4 targets (fourcore_find_v4.cu's find3 shape):
    base = (f d)^6 + 42^6 (c1^6 + c2^6 + c3^6), c1 < c2 < c3 <= N, one residue
    of d and fmax = d; returns (cls, B, d, (c1, c2, c3), base)."""
    rng = np.random.RandomState(seed)
    out = []
    while len(out) < n:
        cls = int(rng.choice([2, 3, 4]))
        B = int(rng.randint(B_lo, B_hi + 1))
        d = int(rng.randint(1, (B - 1) // FREE[cls] + 1))
        c = sorted(int(x) for x in rng.choice(np.arange(1, N + 1), 3, replace=False))
        T = sum(x**6 for x in c)
        if 3 * c[2] ** 6 < T:          # outside the find3 window rule (3 c3^6 >= T)
            continue
        out.append((cls, B, d, tuple(c), (FREE[cls] * d) ** 6 + M42 * T))
    return out


def mixed_unit_array(units, plants5: List[Plant], plants2_4, N: int):
    """One s615_unit array: the mixed units, then class-5 plants, then class
    2-4 plants (all with lim = N)."""
    n = len(units) + len(plants5) + len(plants2_4)
    arr = (s615.Unit * max(n, 1))()
    for i, (c, B, u) in enumerate(units):
        arr[i].cls, arr[i].kind, arr[i].B, arr[i].u = c, 0, B, u
    k = len(units)
    for p in plants5:
        arr[k] = plant_unit(p, N)
        k += 1
    for (cls, B, d, _, base) in plants2_4:
        arr[k] = s615.make_plant234(cls, base, d, lim=N, B=B)
        k += 1
    return arr, n
