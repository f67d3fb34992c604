"""Spreading the transport path over several GPUs, one process per GPU.

The path has no exchange between substrates (every statement of the
reference's step is elementwise in the substrate index: BioFVM_solvers.cpp
:175-273, BioFVM_microenvironment.cpp:595-610, BioFVM_basic_agent.cpp:
234-235) nor between independent microenvironments, so it shards with no
collective inside a step:

* by substrate: rank r owns a contiguous block of substrates of one
  microenvironment (``substrate_range``, ``shard_by_substrate``) and steps
  it alone; the field is assembled only when it is read
  (``gather_substrates``, an all-gather over the process group: NCCL over
  NVLink on GPUs, gloo on CPUs);
* by instance: whole microenvironments are assigned to ranks, balanced by
  their voxel-substrate counts (``assign_instances``).

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
