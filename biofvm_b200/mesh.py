"""Host-side Cartesian mesh geometry, mirroring BioFVM's Cartesian_Mesh.

Pure arithmetic on the host (no device work): node counts, voxel centres,
voxel indices and nearest-voxel lookup, with the reference's exact formulas so
that agents land in the same voxels as in the reference.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def nodes_from_spacing(start: float, end: float, d: float) -> int:
    """(int) ceil(1e-16 + (end - start)/d)  (BioFVM_mesh.cpp:802-805)."""
    return int(math.ceil(1e-16 + (end - start) / d))


@dataclass(frozen=True)
class CartesianMesh:
    """Cartesian_Mesh after resize(x0,x1,y0,y1,z0,z1,dx,dy,dz) (BioFVM_mesh.cpp:796-922)."""

    x0: float
    x1: float
    y0: float
    y1: float
    z0: float
    z1: float
    dx: float
    dy: float
    dz: float

    @property
    def nx(self) -> int:
        return nodes_from_spacing(self.x0, self.x1, self.dx)

    @property
    def ny(self) -> int:
        return nodes_from_spacing(self.y0, self.y1, self.dy)

    @property
    def nz(self) -> int:
        return nodes_from_spacing(self.z0, self.z1, self.dz)

    @property
    def shape(self) -> tuple[int, int, int]:
        return self.nx, self.ny, self.nz

    @property
    def num_voxels(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def dV(self) -> float:
        return self.dx * self.dy * self.dz

    @property
    def uniform(self) -> bool:
        # BioFVM_mesh.cpp:813-815
        tol = 1e-16
        return not (abs(self.dx - self.dy) > tol or abs(self.dy - self.dz) > tol
                    or abs(self.dx - self.dz) > tol)

    def coordinates(self):
        """Voxel centres start + (i + 0.5)*d per axis (BioFVM_mesh.cpp:817-822)."""
        xs = self.x0 + (np.arange(self.nx) + 0.5) * self.dx
        ys = self.y0 + (np.arange(self.ny) + 0.5) * self.dy
        zs = self.z0 + (np.arange(self.nz) + 0.5) * self.dz
        return xs, ys, zs

    def voxel_index(self, i, j, k):
        """(k*ny + j)*nx + i  (BioFVM_mesh.cpp:641-644)."""
        return (np.asarray(k, np.int64) * self.ny + j) * self.nx + i

    def cartesian_indices(self, n):
        n = np.asarray(n, np.int64)
        return n % self.nx, (n // self.nx) % self.ny, n // (self.nx * self.ny)

    def is_position_valid(self, pos: np.ndarray) -> np.ndarray:
        """General_Mesh::is_position_valid (BioFVM_mesh.cpp:208-217)."""
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        lo = np.array([self.x0, self.y0, self.z0])
        hi = np.array([self.x1, self.y1, self.z1])
        return np.all((pos >= lo) & (pos <= hi), axis=1)

    def nearest_voxel_index(self, pos: np.ndarray) -> np.ndarray:
        """floor((x - min)/d) clamped per axis (BioFVM_mesh.cpp:930-948)."""
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        i = np.floor((pos[:, 0] - self.x0) / self.dx).astype(np.int64)
        j = np.floor((pos[:, 1] - self.y0) / self.dy).astype(np.int64)
        k = np.floor((pos[:, 2] - self.z0) / self.dz).astype(np.int64)
        i = np.clip(i, 0, self.nx - 1)
        j = np.clip(j, 0, self.ny - 1)
        k = np.clip(k, 0, self.nz - 1)
        return (k * self.ny + j) * self.nx + i

    def boundary_voxels(self) -> np.ndarray:
        """Indices of every voxel on the mesh boundary, ascending."""
        nx, ny, nz = self.shape
        i = np.arange(nx)
        j = np.arange(ny)
        k = np.arange(nz)
        K, J, I = np.meshgrid(k, j, i, indexing="ij")
        on = (I == 0) | (I == nx - 1) | (J == 0) | (J == ny - 1) | (K == 0) | (K == nz - 1)
        return np.flatnonzero(on.ravel()).astype(np.int64)


def agent_constants(dt: float, volume: np.ndarray, voxel_volume: float, secretion: np.ndarray,
                    saturation: np.ndarray, uptake: np.ndarray):
    """Basic_Agent::set_internal_uptake_constants (BioFVM_basic_agent.cpp:114-148).

    Vectorised over agents, same IEEE operations in the same order:
    c = dt*V/V_voxel; temp1 = ((0 + S)*T)*c; temp2 = (1 + c*S) + c*U.
    """
    volume = np.asarray(volume, np.float64).reshape(-1, 1)
    c = dt * volume / voxel_volume
    t1 = np.zeros_like(secretion, dtype=np.float64)
    t1 = t1 + secretion
    t1 = t1 * saturation
    t1 = t1 * c
    t2 = np.ones_like(secretion, dtype=np.float64)
    t2 = t2 + c * secretion
    t2 = t2 + c * uptake
    return np.ascontiguousarray(t1), np.ascontiguousarray(t2)
