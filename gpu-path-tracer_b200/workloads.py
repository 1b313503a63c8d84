"""Seeded job mixes of the multi-job workloads: batched uneven jobs and open-loop served arrivals.

Batched: 64 independent render jobs over 4 resident sphere-field scenes (10k, 200k, 1.31M and 2M
triangles). Each job draws its resolution log-uniform between 256x256 and 1920x1080, its samples
per pixel uniform in {1, 4, 16, 64}, its path depth uniform in 8..12, and its own camera: a seeded
position on a sphere around the scene centre, looking at the centre.

Served: open-loop Poisson arrivals at a given rate over 8 resident scenes of 50k to 4M triangles;
one seeded job list for every rate (only the arrival times scale with 1/rate). Each job draws its resolution log-uniform between 128x128 and 2048x2048, its samples per pixel from
{4, 16, 64, 256}, its depth uniform in 8..12 and a random camera as above.

The reference renders one job at a time (Renderer::StartSimulation, Renderer.cpp:330-466); these
mixes exercise the job server (gpt_server_*) against that one-job-at-a-time loop.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

import scenes

BATCH_SCENES = ("spheres-10k", "spheres-200k", "spheres-1m", "spheres-2m")
SERVE_SCENES = ("spheres-50k", "spheres-100k", "spheres-250k", "spheres-500k", "spheres-1m", "spheres-2m",
                "spheres-3m", "spheres-4m")
BATCH_SEED = 1002
SERVE_SEED = 1005


@dataclass
class Job:
    scene: str
    width: int
    height: int
    spp: int
    depth: int
    camera: np.ndarray   # 12 floats: origin, lower-left corner, horizontal, vertical
    arrival_s: float = 0.0

    @property
    def paths(self) -> int:
        spa = int(math.isqrt(self.spp))
        return spa * spa * self.width * self.height


def orbit_camera(rng: np.random.Generator, width: int, height: int, box: float = 20.0) -> np.ndarray:
    """A camera on a sphere of radius 0.9 box around the centre of the sphere field (box/2, box/4,
    box/2), at an elevation of 10 to 60 degrees, looking at the centre, 45-degree vertical field of view."""
    center = np.array([0.5 * box, 0.25 * box, 0.5 * box])
    azimuth = rng.uniform(0.0, 2.0 * math.pi)
    elevation = math.radians(rng.uniform(10.0, 60.0))
    radius = 0.9 * box
    pos = center + radius * np.array([math.cos(elevation) * math.cos(azimuth), math.sin(elevation),
                                      math.cos(elevation) * math.sin(azimuth)])
    return scenes.make_camera(tuple(pos), tuple(center), 45.0, width / height)


def log_uniform_resolution(rng: np.random.Generator, lo: tuple[int, int], hi: tuple[int, int]) -> tuple[int, int]:
    """Width and height interpolated geometrically between lo and hi with one uniform draw (the
    pixel count is log-uniform between the two)."""
    t = rng.uniform(0.0, 1.0)
    w = int(round(lo[0] * (hi[0] / lo[0]) ** t))
    h = int(round(lo[1] * (hi[1] / lo[1]) ** t))
    return max(w, 1), max(h, 1)


def batched_jobs(n_jobs: int = 64, seed: int = BATCH_SEED) -> list[Job]:
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n_jobs):
        scene = BATCH_SCENES[int(rng.integers(0, len(BATCH_SCENES)))]
        w, h = log_uniform_resolution(rng, (256, 256), (1920, 1080))
        spp = int(rng.choice([1, 4, 16, 64]))
        depth = int(rng.integers(8, 13))
        jobs.append(Job(scene, w, h, spp, depth, orbit_camera(rng, w, h)))
    return jobs


def served_jobs(rate: float, n_jobs: int, seed: int = SERVE_SEED) -> list[Job]:
    """n_jobs arrivals of a Poisson process of `rate` jobs per second (exponential gaps). The jobs
    themselves and the unit-mean gaps come from the seed alone, and the gaps are divided by the rate,
    so every rate serves the same job list and only the offered load changes."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0, n_jobs)
    t = np.cumsum(gaps) / rate
    jobs = []
    for k in range(n_jobs):
        scene = SERVE_SCENES[int(rng.integers(0, len(SERVE_SCENES)))]
        w, h = log_uniform_resolution(rng, (128, 128), (2048, 2048))
        spp = int(rng.choice([4, 16, 64, 256]))
        depth = int(rng.integers(8, 13))
        jobs.append(Job(scene, w, h, spp, depth, orbit_camera(rng, w, h), arrival_s=float(t[k])))
    return jobs


def percentile(values, q: float) -> float:
    """Nearest-rank percentile (q in [0, 100])."""
    v = sorted(values)
    if not v:
        return float("nan")
    k = max(0, min(len(v) - 1, int(math.ceil(q / 100.0 * len(v))) - 1))
    return float(v[k])
