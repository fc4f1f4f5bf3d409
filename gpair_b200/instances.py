"""Seeded sets of independent reconstruction problems with uneven sizes (the
many-instance workload): image widths drawn from {64, 128, 192, 256}, uv counts
in 500-8,000, triangles = 2/3 of the uv count.

A 4-telescope array observed in 8 channels gives 6 baselines x 8 = 48 V2 points
and 4 triangles x 8 = 32 closure triangles per hour angle, so the uv count is
48 x (hour angles), from 480 to 8,016, with exactly 2/3 as many triangles
(the indexer adds a few uv points where a triangle vertex misses its V2
baseline by more than the reference's matching tolerance).
Each instance draws its scene (1-10 Gaussians / disks / points, unit flux),
array (4 telescopes uniform in a 330 m disk), hour-angle count and noise
from its own seed.
"""
from __future__ import annotations

from typing import List

import numpy as np

from . import api
from .synth import ArrayConfig, make_oifits
from .warmstart import training_scene

WIDTHS = (64, 128, 192, 256)
FIELD_MAS = 6.4


def instance(seed: int) -> api.Problem:
    ss = np.random.SeedSequence(seed)
    s_size, s_scene, s_obs, s_noise = ss.spawn(4)
    r = np.random.default_rng(s_size)
    width = int(r.choice(WIDTHS))
    n_uv = int(r.integers(500, 8001))
    n_ha = max(10, int(round(n_uv / 48)))
    cfg = ArrayConfig(4, 330.0, n_ha, list(np.linspace(1.45e-6, 1.85e-6, 8)), "all")
    scene = training_scene(np.random.default_rng(s_scene), FIELD_MAS)
    oi = make_oifits(cfg, scene, int(s_obs.generate_state(1)[0]), int(s_noise.generate_state(1)[0]))
    return api.problem_from_oifits(oi, width, FIELD_MAS / width, 1e-3)


def instances(n: int, seed0: int = 20_000_000) -> List[api.Problem]:
    return [instance(seed0 + k) for k in range(n)]
