"""Python view of one device-resident Microenvironment, over the C ABI.

Method names follow BioFVM's Microenvironment (BioFVM_microenvironment.h:45-228);
every call goes through libbfvm.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import call, dptr, lptr
from .mesh import CartesianMesh


class Solver:
    """One Microenvironment resident on one GPU (C handle ``bfvm_solver*``)."""

    def __init__(self, device: int = 0):
        _abi.load_library()
        h = ctypes.c_void_p()
        call("bfvm_create", ctypes.byref(h), device)
        self._h = h
        self.device = device
        self._in_flight = []  # host arrays of asynchronous transfers not yet waited for

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if self._h is not None:
            call("bfvm_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- mesh and densities -------------------------------------------------
    def resize_space(self, x0, x1, y0, y1, z0, z1, dx, dy=None, dz=None) -> None:
        dy = dx if dy is None else dy
        dz = dx if dz is None else dz
        call("bfvm_resize_space", self._h, x0, x1, y0, y1, z0, z1, dx, dy, dz)

    def resize_space_uniform(self, x0, x1, y0, y1, z0, z1, dx) -> None:
        self.resize_space(x0, x1, y0, y1, z0, z1, dx, dx, dx)

    def resize_space_nodes(self, x0, x1, y0, y1, z0, z1, nx, ny, nz) -> None:
        call("bfvm_resize_space_nodes", self._h, x0, x1, y0, y1, z0, z1, nx, ny, nz)

    def mesh_info(self):
        nxyz = (ctypes.c_int * 3)()
        geom = (ctypes.c_double * 10)()
        flags = (ctypes.c_int * 2)()
        call("bfvm_get_mesh", self._h, nxyz, geom, flags)
        return tuple(nxyz), tuple(geom), tuple(flags)

    @property
    def shape(self):
        return self.mesh_info()[0]

    @property
    def num_voxels(self) -> int:
        nx, ny, nz = self.shape
        return nx * ny * nz

    def resize_densities(self, n: int) -> None:
        call("bfvm_resize_densities", self._h, n)

    def add_density(self, diffusion_coefficient=0.0, decay_rate=0.0) -> None:
        call("bfvm_add_density", self._h, diffusion_coefficient, decay_rate)

    def set_density(self, index: int, diffusion_coefficient: float, decay_rate: float) -> None:
        call("bfvm_set_density_coefficients", self._h, index, diffusion_coefficient, decay_rate)

    def set_coefficients(self, D, decay) -> None:
        for s, (d, l) in enumerate(zip(np.asarray(D, float), np.asarray(decay, float))):
            self.set_density(s, float(d), float(l))

    @property
    def number_of_densities(self) -> int:
        n = ctypes.c_int()
        call("bfvm_get_num_densities", self._h, ctypes.byref(n))
        return n.value

    def set_densities(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float64)
        assert p.size == self.num_voxels * self.number_of_densities
        call("bfvm_set_densities", self._h, dptr(p))

    def get_densities(self, out: np.ndarray | None = None) -> np.ndarray:
        S = self.number_of_densities
        if out is None:
            out = np.empty((self.num_voxels, S), np.float64)
        call("bfvm_get_densities", self._h, dptr(out))
        return out

    def get_voxel_densities(self, voxels) -> np.ndarray:
        v = np.ascontiguousarray(voxels, np.int64)
        out = np.empty((v.size, self.number_of_densities), np.float64)
        call("bfvm_get_voxel_densities", self._h, v.size, lptr(v), dptr(out))
        return out

    def set_voxel_densities(self, voxels, values) -> None:
        v = np.ascontiguousarray(voxels, np.int64)
        x = np.ascontiguousarray(values, np.float64)
        call("bfvm_set_voxel_densities", self._h, v.size, lptr(v), dptr(x))

    def device_pointer(self) -> int:
        p = ctypes.c_void_p()
        call("bfvm_device_densities", self._h, ctypes.byref(p))
        return p.value or 0

    # -- sources, sinks, boundary -------------------------------------------
    def set_bulk_rates(self, supply=None, target=None, uptake=None) -> None:
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        s, t, u = f(supply), f(target), f(uptake)
        call("bfvm_set_bulk_rates", self._h, dptr(s), dptr(t), dptr(u))

    def set_bulk_rates_sparse(self, voxels, supply=None, target=None, uptake=None) -> None:
        v = np.ascontiguousarray(voxels, np.int64)
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        s, t, u = f(supply), f(target), f(uptake)
        call("bfvm_set_bulk_rates_sparse", self._h, v.size, lptr(v), dptr(s), dptr(t), dptr(u))

    def add_dirichlet_node(self, voxel: int, value) -> None:
        x = np.ascontiguousarray(value, np.float64)
        call("bfvm_add_dirichlet_node", self._h, int(voxel), dptr(x))

    def update_dirichlet_node(self, voxel: int, value) -> None:
        x = np.ascontiguousarray(value, np.float64)
        call("bfvm_update_dirichlet_node", self._h, int(voxel), dptr(x))

    def remove_dirichlet_node(self, voxel: int) -> None:
        call("bfvm_remove_dirichlet_node", self._h, int(voxel))

    def clear_dirichlet_nodes(self) -> None:
        call("bfvm_clear_dirichlet_nodes", self._h)

    def add_dirichlet_nodes(self, voxels, values) -> None:
        values = np.ascontiguousarray(values, np.float64)
        for v, x in zip(np.asarray(voxels, np.int64), values):
            self.add_dirichlet_node(int(v), x)

    def set_agents(self, voxels, temp1, temp2) -> None:
        v = np.ascontiguousarray(voxels, np.int64)
        a = np.ascontiguousarray(temp1, np.float64)
        b = np.ascontiguousarray(temp2, np.float64)
        call("bfvm_set_agents", self._h, v.size, lptr(v), dptr(a), dptr(b))

    def get_agent_densities(self, out: np.ndarray) -> np.ndarray:
        call("bfvm_get_agent_densities", self._h, dptr(out))
        return out

    def set_agents_async(self, voxels, temp1, temp2) -> None:
        """bfvm_set_agents_async: returns at once; steps enqueued afterwards use
        these agents.  The arrays (page-locked, for the copies to overlap the
        steps) are held until wait_transfers() or synchronize()."""
        v = np.ascontiguousarray(voxels, np.int64)
        a = np.ascontiguousarray(temp1, np.float64)
        b = np.ascontiguousarray(temp2, np.float64)
        call("bfvm_set_agents_async", self._h, v.size, lptr(v), dptr(a), dptr(b))
        self._in_flight.extend((v, a, b))

    def get_agent_densities_async(self, out: np.ndarray) -> np.ndarray:
        """bfvm_get_agent_densities_async into out ([A][S] float64, C order),
        which holds the densities after wait_transfers() or synchronize()."""
        if out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-ordered float64 array")
        call("bfvm_get_agent_densities_async", self._h, dptr(out))
        self._in_flight.append(out)
        return out

    def wait_transfers(self) -> None:
        call("bfvm_wait_transfers", self._h)
        self._in_flight.clear()

    # -- stepping -------------------------------------------------------------
    def simulate_bulk_sources_and_sinks(self, dt: float) -> None:
        call("bfvm_simulate_bulk_sources_and_sinks", self._h, dt)

    def simulate_cell_sources_and_sinks(self, dt: float) -> None:
        call("bfvm_simulate_cell_sources_and_sinks", self._h, dt)

    def simulate_diffusion_decay(self, dt: float) -> None:
        call("bfvm_simulate_diffusion_decay", self._h, dt)

    def simulate_diffusion_decay_2d(self, dt: float) -> None:
        call("bfvm_simulate_diffusion_decay_2d", self._h, dt)

    def apply_dirichlet_conditions(self) -> None:
        call("bfvm_apply_dirichlet_conditions", self._h)

    def step(self, dt: float, nsteps: int = 1, flags: int = _abi.STEP_ALL) -> None:
        call("bfvm_step", self._h, dt, nsteps, flags)

    def reset_diffusion_setup(self) -> None:
        call("bfvm_reset_diffusion_setup", self._h)

    # -- gradients (Microenvironment::compute_all_gradient_vectors) -----------
    def compute_all_gradient_vectors(self) -> None:
        call("bfvm_compute_all_gradient_vectors", self._h)

    def get_gradient_vectors(self) -> np.ndarray:
        """[N, S, 3] FP64."""
        out = np.empty((self.num_voxels, self.number_of_densities, 3))
        call("bfvm_get_gradient_vectors", self._h, dptr(out))
        return out

    def set_precision(self, bits: int) -> None:
        call("bfvm_set_precision", self._h, bits)

    def tune_sweeps(self, dt: float, reps: int = 5):
        """Picks each axis's fastest sweep kernel by timing them on this field
        (which is restored); returns [(kernel, chunk, columns, min_blocks,
        row-kernel ring stages)] per axis."""
        call("bfvm_tune_sweeps", self._h, dt, reps)
        out = []
        for ax in range(3):
            k = ctypes.c_int()
            call("bfvm_get_sweep_kernel", self._h, ax, ctypes.byref(k))
            cfg = (ctypes.c_int * 4)()
            call("bfvm_get_sweep_config", self._h, ax, cfg)
            out.append((k.value, cfg[0], cfg[1], cfg[2], cfg[3]))
        return out

    def get_sweep_kernel(self, axis: int) -> int:
        """The kernel `axis` sweeps with under PATH_AUTO: 0 for the default
        (the register kernel), else a PATH_* value."""
        k = ctypes.c_int()
        call("bfvm_get_sweep_kernel", self._h, axis, ctypes.byref(k))
        return k.value

    def set_sweep_config(self, axis: int, chunk: int, columns: int, min_blocks: int = 1) -> None:
        call("bfvm_set_sweep_config", self._h, axis, chunk, columns, min_blocks)

    def get_sweep_config(self, axis: int):
        """(chunk, columns, min_blocks, row-kernel ring stages) of `axis`."""
        cfg = (ctypes.c_int * 4)()
        call("bfvm_get_sweep_config", self._h, axis, cfg)
        return tuple(cfg)

    def set_row_stages(self, stages: int) -> None:
        """Tiles in the x row kernel's shared-memory ring: 2 or 3."""
        call("bfvm_set_row_stages", self._h, stages)

    def set_row_build(self, build: int) -> None:
        """Build of the x row kernel: 0 any density count, 1 a build for this
        density count, 2 (default) the same reading planar chunk tables
        (FP64, 4, 8, 10 or 16 densities; elsewhere build 0 runs)."""
        call("bfvm_set_row_build", self._h, build)

    def get_row_build(self):
        """(requested, effective) row-kernel build."""
        req, eff = ctypes.c_int(), ctypes.c_int()
        call("bfvm_get_row_build", self._h, ctypes.byref(req), ctypes.byref(eff))
        return req.value, eff.value

    def set_kernel_path(self, path: int) -> None:
        call("bfvm_set_kernel_path", self._h, path)

    def set_fuse_sources(self, fuse: bool) -> None:
        call("bfvm_set_fuse_sources", self._h, 1 if fuse else 0)

    def get_fuse_sources(self) -> bool:
        f = ctypes.c_int()
        call("bfvm_get_fuse_sources", self._h, ctypes.byref(f))
        return bool(f.value)

    def synchronize(self) -> None:
        call("bfvm_synchronize", self._h)
        self._in_flight.clear()

    @property
    def stream(self) -> int:
        p = ctypes.c_void_p()
        call("bfvm_get_stream", self._h, ctypes.byref(p))
        return p.value or 0

    @property
    def launch_count(self) -> int:
        n = ctypes.c_int64()
        call("bfvm_get_launch_count", self._h, ctypes.byref(n))
        return n.value

    def set_grid_steps(self, enable: bool) -> None:
        """Whole steps of a small FP64 field (<= 2^19 voxel-densities, <= 64
        points per axis) in one cooperative launch under PATH_AUTO (on by
        default); False gives back the sweep kernels."""
        call("bfvm_set_grid_steps", self._h, 1 if enable else 0)

    def get_grid_steps(self) -> int:
        """Blocks of the cooperative launch bfvm_step would use now (0: none)."""
        b = ctypes.c_int()
        call("bfvm_get_grid_steps", self._h, ctypes.byref(b))
        return b.value

    def set_cluster_steps(self, enable: bool) -> None:
        """Whole steps of a small field in one thread-block cluster (on by
        default under the AUTO kernel path)."""
        call("bfvm_set_cluster_steps", self._h, 1 if enable else 0)

    def get_cluster_steps(self) -> int:
        """Blocks of the cluster that bfvm_step would use now (0: none)."""
        b = ctypes.c_int()
        call("bfvm_get_cluster_steps", self._h, ctypes.byref(b))
        return b.value

    def set_slab_planes(self, planes: int) -> None:
        """x and y sweeps by slabs of `planes` z planes (0: whole axes)."""
        call("bfvm_set_slab_planes", self._h, planes)

    def get_slab_planes(self) -> int:
        k = ctypes.c_int()
        call("bfvm_get_slab_planes", self._h, ctypes.byref(k))
        return k.value

    def profile_step(self, dt: float, nsteps: int, flags: int = _abi.STEP_ALL):
        """(sources, x, y, z) milliseconds per step."""
        ms = (ctypes.c_double * 4)()
        call("bfvm_profile_step", self._h, dt, nsteps, flags, ms)
        return tuple(ms)


def selftest_bounded_wait(device: int = 0, limit_ns: int = 2_000_000):
    """Runs the error path of the TMA sweeps' bounded waits on `device`: a
    kernel waits on a barrier that nothing completes and gives up after
    limit_ns.  Returns (gave_up, waited_ms); the device stays usable."""
    _abi.load_library()
    g = ctypes.c_int()
    ms = ctypes.c_double()
    call("bfvm_selftest_bounded_wait", device, limit_ns, ctypes.byref(g), ctypes.byref(ms))
    return bool(g.value), ms.value


def load_scenario(sv: Solver, scn) -> None:
    """Sets a Solver up from a workloads.Scenario, the way a reference driver
    would: resize, densities and coefficients, initial field, bulk rates,
    Dirichlet nodes in order, agents in creation order."""
    mesh: CartesianMesh = scn.mesh
    sv.resize_densities(scn.S)
    sv.resize_space(mesh.x0, mesh.x1, mesh.y0, mesh.y1, mesh.z0, mesh.z1, mesh.dx, mesh.dy,
                    mesh.dz)
    sv.set_coefficients(scn.D, scn.decay)
    if scn.p0 is not None:
        sv.set_densities(scn.p0)
    if scn.bulk_voxels is not None and len(scn.bulk_voxels):
        sv.set_bulk_rates_sparse(scn.bulk_voxels, scn.bulk_supply, scn.bulk_target,
                                 scn.bulk_uptake)
    if scn.dirichlet_voxels is not None and len(scn.dirichlet_voxels):
        sv.add_dirichlet_nodes(scn.dirichlet_voxels, scn.dirichlet_values)
    if scn.num_agents:
        v, t1, t2 = scn.agent_arrays()
        sv.set_agents(v, t1, t2)
