"""Seeded synthetic SPM workloads (the benchmark configurations).

The reference draws initial positions with an unseeded rand() and a 1.05
sigma overlap test (init_particle.cxx:28-49); the workloads here use the
user_specify route instead (init_particle.cxx:226-288): uniform-random
non-overlapping centres from a PCG64 stream with a stated seed, so that the
GPU path and the reference see the same inputs.
"""
from __future__ import annotations

import numpy as np


def place_spheres(n: int, box, a: float, min_gap: float, seed: int, max_tries: int = 20_000_000) -> np.ndarray:
    """n centres in a periodic box, pairwise centre distance >= 2a + min_gap
    under the minimum image (PCG64(seed), rejection sampling: each draw is
    kept unless it is too close to a centre already kept).  A draw is
    checked against the kept centres in the neighbouring cells of a grid at
    least 2a + min_gap wide, which decides as a check against all would."""
    import itertools

    rng = np.random.Generator(np.random.PCG64(seed))
    box = np.asarray(box, dtype=np.float64)
    dmin = 2 * a + min_gap
    dmin2 = dmin ** 2
    nc = np.maximum(1, np.floor(box / dmin).astype(int))
    grid: dict = {}
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"cannot place {n} spheres of radius {a} in {tuple(box)}")
        c = rng.random(3) * box
        ci = np.minimum((c / box * nc).astype(int), nc - 1)
        axes = [sorted({(int(ci[d]) + o) % int(nc[d]) for o in (-1, 0, 1)}) for d in range(3)]
        near = [k for key in itertools.product(*axes) for k in grid.get(key, ())]
        if near:
            d = np.asarray([pts[k] for k in sorted(near)]) - c
            d -= np.rint(d / box) * box
            if np.min(np.einsum("ij,ij->i", d, d)) < dmin2:
                continue
        grid.setdefault(tuple(int(v) for v in ci), []).append(len(pts))
        pts.append(c)
    return np.asarray(pts, dtype=np.float64).reshape(-1, 3)


def spm_config(np_xyz, n_particles: int, seed: int, a: float = 5.0, a_xi: float = 2.0, kbt: float = 0.0,
               dt: float = 0.01, min_gap: float = 1.0, **extra) -> dict:
    """A Navier_Stokes SPM configuration dict (UDF values of one species)."""
    N = [1 << int(p) for p in np_xyz]
    xs = place_spheres(n_particles, N, a, min_gap, seed) if n_particles else np.zeros((0, 3))
    cfg = {"eq": "Navier_Stokes", "np_xyz": tuple(int(p) for p in np_xyz), "a": a, "a_xi": a_xi, "kbt": kbt,
           "dt": dt, "particles": [{"x": tuple(float(c) for c in x)} for x in xs]}
    cfg.update(extra)
    return cfg


def mixed_128_256() -> dict:
    """128^3, 256 spheres a=5, xi=2 (volume fraction ~0.13), kBT=1e-3 thermal
    kicks, dt=0.01, positions from PCG64 seed 2 with a minimum surface gap of 1."""
    return spm_config((7, 7, 7), 256, seed=2, kbt=1e-3)


def plain_64_16() -> dict:
    """64^3, 16 spheres a=5, xi=2, kBT=0, dt=0.01, seed 1, body force 1e-3 along
    -z applied as gravity with MASS_RATIO = 1 + 1e-3 (md_force.cxx:181-191)."""
    import math

    eps = 1e-3
    g = 1e-3 / (4.0 / 3.0 * math.pi * 5.0 ** 3 * eps)
    return spm_config((6, 6, 6), 16, seed=1, kbt=0.0, gravity_g=g, mass_ratio=1.0 + eps, gravity_dir="-Z")


def electrolyte_128_64() -> dict:
    """128^3, 64 spheres a=5 with surface charge -100 in a monovalent salt
    (Debye length 4, Bjerrum length 0.7 at kBT=1), external field 0.05 along x,
    dt=0.01, positions from PCG64 seed 3."""
    import math

    cfg = spm_config((7, 7, 7), 64, seed=3, kbt=1.0)
    cfg["eq"] = "Electrolyte"
    cfg["alpha_v"] = 0.0
    cfg["alpha_o"] = 0.0
    cfg["electrolyte"] = dict(dielectric=1.0 / (4.0 * math.pi * 0.7), surface_charge=-100.0, debye=4.0,
                              val_p=1.0, val_n=-1.0, onsager_p=1.0, onsager_n=1.0, efield=(0.05, 0.0, 0.0))
    return cfg


def shear_le_128_256() -> dict:
    """The C2 suspension (128^3, 256 spheres a=5, kBT=1e-3, seed 2) under
    Lees-Edwards shear (Shear_Navier_Stokes_Lees_Edwards, DC shear rate 0.01;
    the wall-to-wall velocity difference is 1.28)."""
    cfg = spm_config((7, 7, 7), 256, seed=2, kbt=1e-3)
    cfg["eq"] = "Shear_Navier_Stokes_Lees_Edwards"
    cfg["shear_rate"] = 0.01
    return cfg


BATCH_SHAPES = [(5, 5, 5), (6, 6, 6), (6, 6, 7), (7, 7, 7)]  # 32^3, 64^3, 64x64x128, 128^3


def batched(n_boxes: int = 48, seed: int = 4, max_fill: float = 0.2) -> list:
    """n_boxes independent boxes with shapes drawn from 32^3, 64^3, 64x64x128
    and 128^3, 1-64 spheres each (capped so that the solid volume fraction
    stays below max_fill; a small box cannot hold 64 spheres), radius a drawn
    from [4, 6], xi=2, kBT=1e-3, all from one PCG64(seed) stream."""
    import math

    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for b in range(n_boxes):
        shape = BATCH_SHAPES[int(rng.integers(len(BATCH_SHAPES)))]
        a = float(np.round(rng.uniform(4.0, 6.0), 3))
        vol = float(np.prod([1 << p for p in shape]))
        cap = max(1, int(max_fill * vol / (4.0 / 3.0 * math.pi * a ** 3)))
        n = int(rng.integers(1, 65))
        n = min(n, cap)
        out.append(spm_config(shape, n, seed=1000 * seed + b, a=a, kbt=1e-3))
    return out


def nearcontact_256_dense() -> dict:
    """256^3 at the deployment density of the learned correction: 8600
    spheres a=5, xi=2 (solid volume fraction 0.268), minimum surface gap
    0.25 = 0.05a, kBT=1e-3, dt=0.01, positions from PCG64 seed 5."""
    return spm_config((8, 8, 8), 8600, seed=5, kbt=1e-3, min_gap=0.25)


def nearcontact_256_2048() -> dict:
    """256^3, 2048 spheres a=5, xi=2 (solid volume fraction 0.064), minimum
    surface gap 0.25 = 0.05a so that pairs reach into the near-contact range,
    kBT=1e-3, dt=0.01, positions from PCG64 seed 5 (the deployment case of the
    learned near-contact correction)."""
    return spm_config((8, 8, 8), 2048, seed=5, kbt=1e-3, min_gap=0.25)
