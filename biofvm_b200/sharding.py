"""Spreading the transport path over several GPUs, one process per GPU.

The path has no exchange between substrates (every statement of the
reference's step is elementwise in the substrate index: BioFVM_solvers.cpp
:175-273, BioFVM_microenvironment.cpp:595-610, BioFVM_basic_agent.cpp:
234-235) nor between independent microenvironments, so it shards with no
collective inside a step (except the z-slab split, which exchanges two
planes per slab per step):

* by substrate: rank r owns a contiguous block of substrates of one
  microenvironment (``substrate_range``, ``shard_by_substrate``) and steps
  it alone with its own Solver (``SubstrateShard``); the field is assembled
  only when it is read, by an all-gather of the ranks' device blocks into
  device memory (``SubstrateShard.gather_device``: NCCL over NVLink, no host
  copy; gloo through host memory when the group is a CPU group).
  ``gather_substrates`` does the same for blocks held in host arrays;
* by instance: whole microenvironments are assigned to ranks, balanced by
  their voxel-substrate counts (``assign_instances``).
* by z slab (``ZSlabShard``): rank r owns a slab of z planes of one
  microenvironment; x and y lines stay inside a slab, and each step ends
  with one exchange: every slab's first and last plane are all-gathered and
  a fix-up kernel joins the slabs' z-line segments (bfvm_zslab_fixup).

Every rank takes the same collective steps in the same order.
"""
from __future__ import annotations

import copy

import numpy as np


def substrate_range(S: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous block [s0, s1) of the S substrates for `rank`; the first
    S % world ranks take one more.  Ranks beyond S get an empty block."""
    if not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    base, extra = divmod(S, world)
    s0 = rank * base + min(rank, extra)
    return s0, s0 + base + (1 if rank < extra else 0)


def shard_by_substrate(scn, world: int, rank: int):
    """The scenario restricted to this rank's substrates: coefficients,
    initial field, bulk rates, Dirichlet values and agent rates keep only
    their columns [s0, s1); geometry, node lists and agent positions are
    shared.  Bulk voxels whose rates vanish on the block are kept (their
    update is the identity there)."""
    s0, s1 = substrate_range(scn.S, world, rank)
    sub = copy.copy(scn)
    sub.S = s1 - s0
    cols = slice(s0, s1)

    def take(a):
        return None if a is None else np.ascontiguousarray(np.asarray(a)[:, cols])

    sub.D = np.asarray(scn.D)[cols].copy()
    sub.decay = np.asarray(scn.decay)[cols].copy()
    sub.p0 = take(scn.p0)
    sub.bulk_supply = take(scn.bulk_supply)
    sub.bulk_target = take(scn.bulk_target)
    sub.bulk_uptake = take(scn.bulk_uptake)
    sub.dirichlet_values = take(scn.dirichlet_values)
    sub.agent_secretion = take(scn.agent_secretion)
    sub.agent_saturation = take(scn.agent_saturation)
    sub.agent_uptake = take(scn.agent_uptake)
    sub.meta = dict(scn.meta, substrates=(s0, s1))
    return sub


def gather_substrates(local: np.ndarray, S: int, group=None) -> np.ndarray:
    """[N, S] field from every rank's [N, s1 - s0] block (all-gather; the
    result is on every rank).  Blocks may be empty."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else \
        torch.device("cpu")
    N = local.shape[0]
    width = max(substrate_range(S, world, r)[1] - substrate_range(S, world, r)[0]
                for r in range(world))
    # equal-sized blocks for the all-gather; each rank fills its own columns
    buf = torch.zeros((N, width), dtype=torch.float64, device=dev)
    if local.shape[1]:
        buf[:, :local.shape[1]] = torch.from_numpy(np.ascontiguousarray(local)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.empty((N, S))
    for r in range(world):
        s0, s1 = substrate_range(S, world, r)
        out[:, s0:s1] = parts[r][:, :s1 - s0].cpu().numpy()
    return out


def assign_instances(sizes, world: int) -> list[int]:
    """Rank of every instance: largest first onto the least-loaded rank
    (ties to the lower rank), so the per-rank voxel-substrate totals are
    balanced.  Deterministic: every rank computes the same assignment."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += int(sizes[i])
    return owner


class _DeviceArray:
    """A raw device allocation seen through __cuda_array_interface__ (no
    copy), for torch.as_tensor."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


class SubstrateShard:
    """This rank's block of substrates of one microenvironment, stepped by a
    Solver on this rank's GPU.  The whole [N, S] field exists only when read:
    ``gather_device`` all-gathers every rank's device block into a device
    tensor (NCCL over NVLink; no host copy), ``gather`` brings that to the
    host.  A rank past the S-th holds no substrates and no Solver, but takes
    part in every collective.  FP64 fields."""

    def __init__(self, scn, device: int = 0, group=None):
        import torch.distributed as dist

        from .solver import Solver, load_scenario

        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.S = scn.S
        self.N = scn.num_voxels
        self.device = device
        self.s0, self.s1 = substrate_range(scn.S, self.world, self.rank)
        self.sub = shard_by_substrate(scn, self.world, self.rank)
        self.solver = None
        if self.sub.S:
            self.solver = Solver(device)
            load_scenario(self.solver, self.sub)

    def close(self) -> None:
        if self.solver is not None:
            self.solver.close()
            self.solver = None

    def step(self, dt: float, nsteps: int = 1, flags: int | None = None) -> None:
        from ._abi import STEP_ALL

        if self.solver is not None:
            self.solver.step(dt, nsteps, STEP_ALL if flags is None else flags)

    def synchronize(self) -> None:
        if self.solver is not None:
            self.solver.synchronize()

    def device_block(self):
        """This rank's [N, s1 - s0] block as a torch tensor over the solver's
        own device memory (valid until the solver is resized or closed)."""
        import torch

        dev = torch.device("cuda", self.device)
        if self.solver is None:
            return torch.empty((self.N, 0), dtype=torch.float64, device=dev)
        return torch.as_tensor(_DeviceArray(self.solver.device_pointer(),
                                            (self.N, self.s1 - self.s0), "<f8"), device=dev)

    def gather_device(self):
        """The whole [N, S] field on this rank's GPU: every rank's block is
        padded to the widest block and all-gathered (NCCL), then the blocks'
        columns are placed side by side on the device."""
        import torch
        import torch.distributed as dist

        self.synchronize()
        dev = torch.device("cuda", self.device)
        width = max(b - a for a, b in (substrate_range(self.S, self.world, r)
                                       for r in range(self.world)))
        block = self.device_block()
        on_gpu = dist.get_backend(self.group) == "nccl"
        cdev = dev if on_gpu else torch.device("cpu")
        send = torch.zeros((self.N, width), dtype=torch.float64, device=cdev)
        send[:, :block.shape[1]] = block
        # the output is the ranks' blocks one after another along the first
        # axis (the form every backend takes)
        recv = torch.empty((self.world * self.N, width), dtype=torch.float64, device=cdev)
        dist.all_gather_into_tensor(recv, send, group=self.group)
        recv = recv.view(self.world, self.N, width)
        out = torch.empty((self.N, self.S), dtype=torch.float64, device=dev)
        for r in range(self.world):
            a, b = substrate_range(self.S, self.world, r)
            out[:, a:b] = recv[r, :, :b - a]
        return out

    def gather(self) -> np.ndarray:
        return self.gather_device().cpu().numpy()


# ---- one field split by z planes ----------------------------------------

def z_bounds(nz: int, world: int) -> list[int]:
    """Plane boundaries of `world` z slabs of nz planes: slab r holds planes
    [b[r], b[r+1]); the first nz % world slabs take one more plane.  Every
    slab needs at least one plane (world <= nz)."""
    if not 1 <= world <= nz:
        raise ValueError("need 1 <= world <= nz")
    return [substrate_range(nz, world, r)[0] for r in range(world)] + [nz]


class ZSlabShard:
    """This rank's slab of z planes of one microenvironment, stepped by a
    Solver on this rank's GPU (bfvm_set_z_slab).  x and y lines lie in one
    plane and are solved by the slab alone; each step's z sweep solves the
    slab's segment of every z line with zero carries at its ends, then every
    slab's first and last plane are all-gathered into device memory (NCCL
    over NVLink; gloo through host memory for a CPU group) and
    bfvm_zslab_fixup joins the segments, so the result equals the unsplit
    solve to rounding.  Bulk entries, Dirichlet nodes and agents go to the
    slab that holds their voxel, in their original order (agents' voxels and
    constants from the whole mesh, so each lands in the reference's voxel).
    FP64 fields."""

    def __init__(self, scn, device: int = 0, group=None):
        import torch.distributed as dist

        from . import _abi
        from .mesh import CartesianMesh
        from .solver import Solver

        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.device = device
        m = scn.mesh
        self.nx, self.ny, self.nz = m.nx, m.ny, m.nz
        self.S = scn.S
        self.plane = self.nx * self.ny
        self.bounds = z_bounds(self.nz, self.world)
        b0, b1 = self.bounds[self.rank], self.bounds[self.rank + 1]
        self.z0, self.z1 = b0, b1
        sm = CartesianMesh(m.x0, m.x1, m.y0, m.y1, m.z0 + b0 * m.dz, m.z0 + b1 * m.dz, m.dx,
                           m.dy, m.dz)
        if sm.nz != b1 - b0:
            raise ValueError("the slab's z extent does not give a whole number of planes")
        lo, hi = b0 * self.plane, b1 * self.plane
        sv = Solver(device)
        sv.resize_densities(scn.S)
        sv.resize_space(sm.x0, sm.x1, sm.y0, sm.y1, sm.z0, sm.z1, sm.dx, sm.dy, sm.dz)
        sv.set_coefficients(scn.D, scn.decay)
        if scn.p0 is not None:
            sv.set_densities(np.ascontiguousarray(np.asarray(scn.p0)[lo:hi]))
        if scn.bulk_voxels is not None and len(scn.bulk_voxels):
            bv = np.asarray(scn.bulk_voxels)
            keep = (bv >= lo) & (bv < hi)
            if keep.any():
                def rows(a):
                    return None if a is None else np.asarray(a)[keep]

                sv.set_bulk_rates_sparse(bv[keep] - lo, rows(scn.bulk_supply),
                                         rows(scn.bulk_target), rows(scn.bulk_uptake))
        if scn.dirichlet_voxels is not None and len(scn.dirichlet_voxels):
            dv = np.asarray(scn.dirichlet_voxels)
            keep = (dv >= lo) & (dv < hi)
            if keep.any():
                sv.add_dirichlet_nodes(dv[keep] - lo, np.asarray(scn.dirichlet_values)[keep])
        if scn.num_agents:
            v, t1, t2 = scn.agent_arrays()
            keep = (v >= lo) & (v < hi)
            if keep.any():
                sv.set_agents(v[keep] - lo, t1[keep], t2[keep])
        _abi.call("bfvm_set_z_slab", sv.handle, self.world, _int_array(self.bounds), self.rank)
        self.solver = sv

    def close(self) -> None:
        if self.solver is not None:
            self.solver.close()
            self.solver = None

    def _field(self):
        import torch

        return torch.as_tensor(_DeviceArray(self.solver.device_pointer(),
                                            (self.z1 - self.z0, self.plane * self.S), "<f8"),
                               device=torch.device("cuda", self.device))

    def step(self, dt: float, nsteps: int = 1, flags: int | None = None) -> None:
        """nsteps steps; each joins the slabs after its z sweep (one
        all-gather of two planes per slab)."""
        import torch
        import torch.distributed as dist

        from . import _abi

        flags = _abi.STEP_ALL if flags is None else flags
        dev = torch.device("cuda", self.device)
        on_gpu = dist.get_backend(self.group) == "nccl"
        C = self.plane * self.S
        stream = torch.cuda.ExternalStream(self.solver.stream, device=dev)
        for _ in range(nsteps):
            self.solver.step(dt, 1, flags)
            if not flags & _abi.STEP_DIFFUSION:
                continue
            # the collective and the copies run on the solver's stream, in
            # order with its kernels
            with torch.cuda.stream(stream):
                f = self._field()
                send = torch.stack([f[0], f[-1]])
                # [world * 2][C]: every slab's first and last plane in rank order
                if on_gpu:
                    recv = torch.empty((self.world * 2, C), dtype=torch.float64, device=dev)
                    dist.all_gather_into_tensor(recv, send, group=self.group)
                else:
                    recv_h = torch.empty((self.world * 2, C), dtype=torch.float64)
                    dist.all_gather_into_tensor(recv_h, send.cpu(), group=self.group)
                    recv = recv_h.to(dev)
                # recv was allocated on this stream: the allocator hands its
                # memory out again only to work ordered after the fix-up
                _abi.call("bfvm_zslab_fixup", self.solver.handle, recv.data_ptr())

    def gather_device(self):
        """The whole [N, S] field on this rank's GPU (all-gather of the slabs,
        padded to the thickest)."""
        import torch
        import torch.distributed as dist

        self.solver.synchronize()
        dev = torch.device("cuda", self.device)
        thick = max(self.bounds[r + 1] - self.bounds[r] for r in range(self.world))
        C = self.plane * self.S
        on_gpu = dist.get_backend(self.group) == "nccl"
        cdev = dev if on_gpu else torch.device("cpu")
        send = torch.zeros((thick, C), dtype=torch.float64, device=cdev)
        send[:self.z1 - self.z0] = self._field()
        recv = torch.empty((self.world * thick, C), dtype=torch.float64, device=cdev)
        dist.all_gather_into_tensor(recv, send, group=self.group)
        recv = recv.view(self.world, thick, C)
        out = torch.empty((self.nz, C), dtype=torch.float64, device=dev)
        for r in range(self.world):
            a, b = self.bounds[r], self.bounds[r + 1]
            out[a:b] = recv[r, :b - a]
        return out.reshape(self.nz * self.plane, self.S)

    def gather(self) -> np.ndarray:
        return self.gather_device().cpu().numpy()


def _int_array(values):
    import ctypes

    return (ctypes.c_int * len(values))(*values)
