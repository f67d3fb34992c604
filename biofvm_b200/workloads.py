"""Seeded synthetic workloads for the transport path (no dataset is involved).

Each builder returns a Scenario: the mesh, the densities' coefficients, the
initial field, bulk rates (sparse: only voxels with non-zero rates), the
Dirichlet nodes in insertion order and the agents in creation order, with
per-agent rates.  The same Scenario drives the GPU library, the compiled
reference and the CPU oracle, so their inputs are identical.

Named workloads (sizes as stated; all seeded):
  plain_50     50^3 voxels (dx=20 on a 1000 um cube), 1 substrate, D=1e5,
               decay 0.1, dt=0.01, 100 steps, Dirichlet 1.0 on all 14,408
               boundary voxels, 1000 uptake agents (V=2494, U=10).
  lod_256      256^3 voxels (dx=10), 10 substrates, D log-uniform [1e3,1e5],
               decay uniform [0.01,1], dt=0.01, 100 steps, bulk supply 0.5 /
               target 1.0 inside a radius-500 sphere at the centre, 100k agents
               (U in [0,10], S in [0,1], saturation 1.0, V=2494).
  batched_64   64 instances, nx,ny,nz in [32,128], S in 1..8, 0-20k agents.
  adjoint_128  128^3, 4 substrates, 20k agents, 200 steps.
  fp32_512     512^3, 8 substrates, 1M agents, 50 steps.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import CartesianMesh, agent_constants

CELL_VOLUME = 2494.0  # um^3, the radius-8.4 um cell of the 1000-agent workload


@dataclass
class Scenario:
    name: str
    mesh: CartesianMesh
    S: int
    D: np.ndarray
    decay: np.ndarray
    dt: float
    steps: int
    p0: np.ndarray | None = None  # [N, S]
    bulk_voxels: np.ndarray | None = None  # [E] ascending
    bulk_supply: np.ndarray | None = None  # [E, S]
    bulk_target: np.ndarray | None = None
    bulk_uptake: np.ndarray | None = None
    dirichlet_voxels: np.ndarray | None = None  # [nd] insertion order
    dirichlet_values: np.ndarray | None = None  # [nd, S]
    agent_pos: np.ndarray | None = None  # [A, 3]
    agent_volume: np.ndarray | None = None  # [A]
    agent_secretion: np.ndarray | None = None  # [A, S]
    agent_saturation: np.ndarray | None = None
    agent_uptake: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return self.mesh.shape

    @property
    def num_voxels(self) -> int:
        return self.mesh.num_voxels

    @property
    def num_agents(self) -> int:
        return 0 if self.agent_pos is None else int(self.agent_pos.shape[0])

    def initial_field(self) -> np.ndarray:
        if self.p0 is not None:
            return np.array(self.p0, np.float64, copy=True)
        return np.zeros((self.num_voxels, self.S), np.float64)

    def agent_arrays(self):
        """(voxel[A], temp1[A,S], temp2[A,S]) as Basic_Agent computes them."""
        vox = self.mesh.nearest_voxel_index(self.agent_pos)
        t1, t2 = agent_constants(self.dt, self.agent_volume, self.mesh.dV, self.agent_secretion,
                                 self.agent_saturation, self.agent_uptake)
        return vox, t1, t2

    def dense_bulk(self):
        """[N, S] supply, target, uptake tables (None where all zero)."""
        if self.bulk_voxels is None or not len(self.bulk_voxels):
            return None, None, None
        out = []
        for a in (self.bulk_supply, self.bulk_target, self.bulk_uptake):
            if a is None:
                out.append(None)
                continue
            d = np.zeros((self.num_voxels, self.S), np.float64)
            d[self.bulk_voxels] = a
            out.append(d)
        return tuple(out)


def _agents(rng, mesh: CartesianMesh, A: int, S: int, uptake_max=10.0, secretion_max=1.0,
            saturation=1.0, volume=CELL_VOLUME):
    lo = np.array([mesh.x0, mesh.y0, mesh.z0])
    hi = np.array([mesh.x1, mesh.y1, mesh.z1])
    pos = lo + rng.random((A, 3)) * (hi - lo)
    up = rng.uniform(0.0, uptake_max, (A, S))
    sec = rng.uniform(0.0, secretion_max, (A, S))
    sat = np.full((A, S), saturation)
    vol = np.full(A, volume)
    return pos, vol, sec, sat, up


def _sphere_bulk(mesh: CartesianMesh, S: int, radius: float, supply: float, target: float):
    xs, ys, zs = mesh.coordinates()
    cx = 0.5 * (mesh.x0 + mesh.x1)
    cy = 0.5 * (mesh.y0 + mesh.y1)
    cz = 0.5 * (mesh.z0 + mesh.z1)
    Z, Y, X = np.meshgrid(zs - cz, ys - cy, xs - cx, indexing="ij")
    inside = (X * X + Y * Y + Z * Z <= radius * radius).ravel()
    vox = np.flatnonzero(inside).astype(np.int64)
    E = vox.size
    return vox, np.full((E, S), supply), np.full((E, S), target), np.zeros((E, S))


def plain_50(steps: int = 100, seed: int = 12346, n_agents: int = 1000) -> Scenario:
    """50^3, 1 substrate, all-boundary Dirichlet 1.0, 1000 uptake agents."""
    rng = np.random.default_rng(seed)
    mesh = CartesianMesh(0.0, 1000.0, 0.0, 1000.0, 0.0, 1000.0, 20.0, 20.0, 20.0)
    S = 1
    dv = mesh.boundary_voxels()
    pos, vol, sec, sat, up = _agents(rng, mesh, n_agents, S)
    up[:] = 10.0
    sec[:] = 0.0
    sat[:] = 0.0
    return Scenario("plain_50", mesh, S, np.array([1e5]), np.array([0.1]), 0.01, steps,
                    p0=None, dirichlet_voxels=dv, dirichlet_values=np.ones((dv.size, S)),
                    agent_pos=pos, agent_volume=vol, agent_secretion=sec,
                    agent_saturation=sat, agent_uptake=up)


def lod_cube(n: int = 256, S: int = 10, n_agents: int = 100_000, steps: int = 100,
             dx: float = 10.0, seed: int = 12347, bulk_radius: float = 500.0,
             name: str | None = None) -> Scenario:
    """n^3 voxels at dx, S substrates, central bulk sphere, uniform agents
    (the 256^3 x 10 headline workload at the defaults)."""
    rng = np.random.default_rng(seed)
    L = n * dx
    mesh = CartesianMesh(0.0, L, 0.0, L, 0.0, L, dx, dx, dx)
    D = np.exp(rng.uniform(np.log(1e3), np.log(1e5), S))
    decay = rng.uniform(0.01, 1.0, S)
    bv, bs, bt, bu = _sphere_bulk(mesh, S, bulk_radius, 0.5, 1.0)
    pos, vol, sec, sat, up = _agents(rng, mesh, n_agents, S)
    return Scenario(name or f"lod_{n}", mesh, S, D, decay, 0.01, steps, bulk_voxels=bv,
                    bulk_supply=bs, bulk_target=bt, bulk_uptake=bu, agent_pos=pos,
                    agent_volume=vol, agent_secretion=sec, agent_saturation=sat,
                    agent_uptake=up)


def lod_256(steps: int = 100) -> Scenario:
    return lod_cube(256, 10, 100_000, steps, name="lod_256")


def mixed_small(shape=(24, 20, 16), S: int = 3, n_agents: int = 600, seed: int = 7,
                dx: float = 10.0, steps: int = 5, dirichlet: bool = True,
                bulk: bool = True, dense_p0: bool = True) -> Scenario:
    """A small non-cubic case exercising every part of the step: random
    initial field, bulk rates (including uptake) on a random subset of voxels,
    a few Dirichlet nodes (one repeated), and agents with many shared voxels."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    mesh = CartesianMesh(0.0, nx * dx, 0.0, ny * dx, 0.0, nz * dx, dx, dx, dx)
    N = mesh.num_voxels
    D = np.exp(rng.uniform(np.log(1e2), np.log(1e5), S))
    decay = rng.uniform(0.0, 1.0, S)
    p0 = rng.uniform(0.0, 2.0, (N, S)) if dense_p0 else None
    sc = Scenario("mixed", mesh, S, D, decay, 0.01, steps, p0=p0)
    if bulk:
        E = max(1, N // 7)
        bv = np.sort(rng.choice(N, E, replace=False)).astype(np.int64)
        sc.bulk_voxels = bv
        sc.bulk_supply = rng.uniform(0.0, 2.0, (E, S))
        sc.bulk_target = rng.uniform(0.0, 3.0, (E, S))
        sc.bulk_uptake = rng.uniform(0.0, 1.0, (E, S))
    if dirichlet:
        nd = max(2, N // 50)
        dv = rng.choice(N, nd, replace=False).astype(np.int64)
        dv = np.concatenate([dv, dv[:1]])  # a repeated node: the later value wins
        sc.dirichlet_voxels = dv
        sc.dirichlet_values = rng.uniform(0.0, 5.0, (dv.size, S))
    if n_agents:
        # cluster agents so that many share a voxel (order matters there)
        pos, vol, sec, sat, up = _agents(rng, mesh, n_agents, S)
        q = n_agents // 4
        hot = pos[:q]
        pos[q: 2 * q] = hot + rng.uniform(-0.1, 0.1, hot.shape)
        pos = np.clip(pos, [mesh.x0, mesh.y0, mesh.z0], [mesh.x1, mesh.y1, mesh.z1])
        vol = rng.uniform(500.0, 4000.0, n_agents)
        sat = rng.uniform(0.0, 2.0, (n_agents, S))
        sc.agent_pos, sc.agent_volume = pos, vol
        sc.agent_secretion, sc.agent_saturation, sc.agent_uptake = sec, sat, up
    return sc


def convergence_1d(dt: float = 0.01, t_max: float = 0.5, dx: float = 20.0) -> Scenario:
    """The 1-D known-answer problem of the reference's convergence test 1
    (examples/convergence_test1.cpp:56-91): x in [-500, 500], one voxel thick
    in y and z, D=1e5, no decay, u0 = 1 + cos(pi*|x|/500)."""
    mesh = CartesianMesh(-500.0, 500.0, -dx / 2, dx / 2, -dx / 2, dx / 2, dx, dx, dx)
    xs, _, _ = mesh.coordinates()
    p0 = (1.0 + np.cos(np.pi / 500.0 * np.abs(xs))).reshape(-1, 1)
    steps = int(round(t_max / dt))
    return Scenario("convergence_1d", mesh, 1, np.array([1e5]), np.array([0.0]), dt, steps,
                    p0=p0, meta={"t_max": steps * dt})


def convergence_1d_exact(scn: Scenario) -> np.ndarray:
    """u(x, t) = 1 + cos(pi x/L0) exp(-D pi^2 t / L0^2), L0 = 500
    (examples/convergence_test1_analytical.cpp:76-84)."""
    xs, _, _ = scn.mesh.coordinates()
    t = scn.meta["t_max"]
    D = float(scn.D[0])
    return 1.0 + np.cos(np.pi / 500.0 * np.abs(xs)) * np.exp(-D * np.pi ** 2 * t / 500.0 ** 2)


def batched_instances(count: int = 64, seed: int = 12348, n_min: int = 32, n_max: int = 128,
                      max_agents: int = 20_000, dx: float = 10.0, steps: int = 200):
    """The independent microenvironments of the batched workload."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(n_min, n_max + 1, 3))
        S = int(rng.integers(1, 9))
        A = int(rng.integers(0, max_agents + 1))
        mesh = CartesianMesh(0.0, nx * dx, 0.0, ny * dx, 0.0, nz * dx, dx, dx, dx)
        D = np.exp(rng.uniform(np.log(1e3), np.log(1e5), S))
        decay = rng.uniform(0.01, 1.0, S)
        bv, bs, bt, bu = _sphere_bulk(mesh, S, 500.0, 0.5, 1.0)
        pos, vol, sec, sat, up = _agents(rng, mesh, A, S)
        out.append(Scenario(f"batch{b}", mesh, S, D, decay, 0.01, steps, bulk_voxels=bv,
                            bulk_supply=bs, bulk_target=bt, bulk_uptake=bu, agent_pos=pos,
                            agent_volume=vol, agent_secretion=sec, agent_saturation=sat,
                            agent_uptake=up))
    return out
