"""Golden cases: each is a seeded Scenario plus the part of the step that is
run (flags: 1 bulk, 2 cells, 4 diffusion) and how many steps.  The outputs
were produced by the UNMODIFIED reference (see make_golden.py)."""
from __future__ import annotations

import hashlib

import numpy as np

from biofvm_b200 import workloads as W

# name -> (builder, flags, steps, store)   store: "full" array or "sha" digest + samples
CASES = {
    "mixed_full": (lambda: W.mixed_small(), 7, 5, "full"),
    "mixed_thin_axis": (lambda: W.mixed_small(shape=(7, 1, 5), S=2, n_agents=50, seed=3), 7, 4,
                        "full"),
    "mixed_odd": (lambda: W.mixed_small(shape=(33, 17, 9), S=4, n_agents=400, seed=11,
                                        dirichlet=False), 7, 3, "full"),
    "small_bulk_only": (lambda: W.mixed_small(shape=(12, 10, 8), seed=21), 1, 2, "full"),
    "small_cells_only": (lambda: W.mixed_small(shape=(12, 10, 8), seed=22, n_agents=300), 2, 2,
                         "full"),
    "small_diffusion_only": (lambda: W.mixed_small(shape=(12, 10, 8), seed=23), 4, 3, "full"),
    "single_voxel": (lambda: W.mixed_small(shape=(1, 1, 1), S=2, n_agents=5, seed=5,
                                           dirichlet=False), 7, 3, "full"),
    "plain_50": (lambda: W.plain_50(), 7, 100, "sha"),
    "lod_20": (lambda: W.lod_cube(20, 5, 500, steps=5, seed=99, bulk_radius=60.0,
                                  name="lod_20"), 7, 5, "sha"),
    "convergence_1d": (lambda: W.convergence_1d(dt=0.01, t_max=0.5), 4, 50, "full"),
}

N_SAMPLES = 2000


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float64).tobytes()).hexdigest()


def input_fingerprint(scn) -> str:
    """Digest of every input array of a Scenario (detects a changed builder)."""
    h = hashlib.sha256()
    h.update(repr((scn.mesh, scn.S, scn.dt, scn.steps)).encode())
    for a in (scn.D, scn.decay, scn.p0, scn.bulk_voxels, scn.bulk_supply, scn.bulk_target,
              scn.bulk_uptake, scn.dirichlet_voxels, scn.dirichlet_values, scn.agent_pos,
              scn.agent_volume, scn.agent_secretion, scn.agent_saturation, scn.agent_uptake):
        h.update(b"-" if a is None else np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def sample_index(size: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(size, min(size, N_SAMPLES), replace=False))
