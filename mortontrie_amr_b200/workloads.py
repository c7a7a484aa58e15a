"""Seeded synthetic workloads of many independent cases.

batched_uneven_cases: the batched-instances workload -- lid-driven cavities
and flows past a sphere of uneven size: coarse domains drawn from 32^3,
64x32x32, 64^3 and 128x64x64, 1 to 3 refinement levels around the body or
under the lid, Re uniform in [10, 200], D3Q19 LBGK or D3Q27 cumulant.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .case import Case, cavity_case, nested_sphere_case

DOMAINS = [(32, 32, 32), (64, 32, 32), (64, 64, 64), (128, 64, 64)]
MODELS = [(19, "LBGK"), (27, "Cumulant")]


@dataclass
class CaseSpec:
    kind: str          # "cavity" or "sphere"
    coarse: tuple
    levels: int        # refinement levels (max_level)
    re: float
    q: int
    collision: str

    def build(self, mesh: str = "host") -> Case:
        if self.kind == "cavity":
            nx, ny, nz = self.coarse
            lo, hi = [2, 2, nz // 2], [nx - 2, ny - 2, nz - 2]
            refine = []
            for l in range(self.levels):
                s = 1 << l
                refine.append((tuple(v * s for v in lo), tuple(v * s for v in hi)))
                lo = [lo[0] + 2, lo[1] + 2, lo[2] + 2]
                hi = [hi[0] - 2, hi[1] - 2, hi[2] - 2]
            return cavity_case(q=self.q, collision=self.collision, coarse=self.coarse, max_level=self.levels,
                               re=self.re, u_lid=0.05, refine=refine, mesh=mesh)
        nx, ny, nz = self.coarse
        r = max(2, ny // 10)
        hw = (3.0, 2.0, 1.4)[: self.levels]
        cx = max(nx // 4, int(np.ceil(hw[0] * r)) + 2)
        return nested_sphere_case(q=self.q, collision=self.collision, coarse=self.coarse, max_level=self.levels,
                                  center=(cx, ny // 2, nz // 2), radius=float(r), half_widths=hw, u=0.05,
                                  re=self.re, mesh=mesh)

    def label(self) -> str:
        return (f"{self.kind} {'x'.join(map(str, self.coarse))} L{self.levels} Re{self.re:.0f} "
                f"D3Q{self.q} {self.collision}")


def batched_uneven_cases(seed: int = 4, n: int = 64) -> list:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        kind = ("cavity", "sphere")[rng.integers(2)]
        coarse = DOMAINS[rng.integers(len(DOMAINS))]
        levels = int(rng.integers(1, 4))
        re = float(rng.uniform(10.0, 200.0))
        q, coll = MODELS[rng.integers(2)]
        out.append(CaseSpec(kind, coarse, levels, re, q, coll))
    return out

